"""gev_poisson_noalloc (static device scratch, no allocation) against the
context's phi update with prepare == 0 (gev_solve_phi) on the same source:
two calls in a row, an in-place call, calls on a side stream, and the size
limit of the scratch.  Collected last so that it also runs after every other
GPU test in the session."""
import numpy as np
import pytest

from _fixtures import rel_err

gev = pytest.importorskip("gevb200")
torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = {gev.FP64: 1e-12, gev.MIXED: 1e-5}


def _source(N, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(N ** 3)


@pytest.mark.parametrize("prec", [gev.FP64, gev.MIXED])
@pytest.mark.parametrize("N", [32, 128])
def test_noalloc_matches_solve_phi(prec, N):
    coeff, modif = 0.37, 0.0 if N == 32 else 1e-3
    src = _source(N, 11 + N)
    with gev.Context(N, precision=prec, capacity=1) as c:
        c.set_field(gev.FIELD_SOURCE, src)
        c.solve_phi(False, 0.0, 0.0, 0.0, 0.0, coeff, modif)
        ref = c.get_field(gev.FIELD_PHI).ravel()
    dt = torch.float64 if prec == gev.FP64 else torch.float32
    d_src = torch.tensor(src, dtype=dt, device="cuda")
    d_phi = torch.empty(N ** 3, dtype=dt, device="cuda")
    for call in range(2):   # two calls in a row reuse the same scratch
        d_phi.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = gev.poisson_noalloc(N, prec, d_src.data_ptr(), d_phi.data_ptr(), coeff, modif)
        assert rc == gev.GEV_OK, rc
        torch.cuda.synchronize()
        out = d_phi.double().cpu().numpy()
        assert np.all(np.isfinite(out)), call
        assert rel_err(out, ref) < TOL[prec], (call, rel_err(out, ref))


@pytest.mark.parametrize("prec", [gev.FP64, gev.MIXED])
def test_noalloc_in_place_and_on_a_stream(prec):
    """phi may be the source array (the first pass copies the source into the
    scratch spectrum before anything is written to phi), and the work follows
    the stream it is given: two calls queued on a side stream, the second in
    place, match solve_phi after that stream is synchronised."""
    N, coeff, modif = 64, 0.91, 2e-3
    src = _source(N, 77)
    with gev.Context(N, precision=prec, capacity=1) as c:
        c.set_field(gev.FIELD_SOURCE, src)
        c.solve_phi(False, 0.0, 0.0, 0.0, 0.0, coeff, modif)
        ref = c.get_field(gev.FIELD_PHI).ravel()
    dt = torch.float64 if prec == gev.FP64 else torch.float32
    side = torch.cuda.Stream()
    d_src = torch.tensor(src, dtype=dt, device="cuda")
    d_phi = torch.full((N ** 3,), float("nan"), dtype=dt, device="cuda")
    d_io = d_src.clone()
    torch.cuda.synchronize()
    rc1 = gev.poisson_noalloc(N, prec, d_src.data_ptr(), d_phi.data_ptr(), coeff, modif, side.cuda_stream)
    rc2 = gev.poisson_noalloc(N, prec, d_io.data_ptr(), d_io.data_ptr(), coeff, modif, side.cuda_stream)
    assert rc1 == gev.GEV_OK and rc2 == gev.GEV_OK, (rc1, rc2)
    side.synchronize()
    for out in (d_phi, d_io):
        o = out.double().cpu().numpy()
        assert np.all(np.isfinite(o))
        assert rel_err(o, ref) < TOL[prec], rel_err(o, ref)


def test_noalloc_rejects_sizes_beyond_scratch():
    d = torch.zeros(8, dtype=torch.float32, device="cuda")
    assert gev.poisson_noalloc(256, gev.MIXED, d.data_ptr(), d.data_ptr(), 1.0, 0.0) == gev.GEV_ERR_SIZE
    assert gev.poisson_noalloc(20, gev.MIXED, d.data_ptr(), d.data_ptr(), 1.0, 0.0) == gev.GEV_ERR_ARG
    assert gev.poisson_noalloc(32, 9, d.data_ptr(), d.data_ptr(), 1.0, 0.0) == gev.GEV_ERR_ARG
    assert gev.poisson_noalloc(32, gev.MIXED, 0, d.data_ptr(), 1.0, 0.0) == gev.GEV_ERR_ARG

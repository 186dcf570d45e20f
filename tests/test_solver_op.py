"""The solvers over an operator given as a callback (lc_cgsolver_op,
lc_split_bregman_op), the reference's opt::Function<T> argument
(include/optimize.h:30-31, 74-91).  The reference's own CG test runs on a
non-Toeplitz operator (tests/test_cg_normal.cpp:47-101); here the NUFFT
normal operator (sysmat2d with the polar grid) through a Python callback
against the FP64 oracle's CG and Split-Bregman on its exact NUDFT operator,
and the Toeplitz operator through a callback against the PSF-handle solver."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

RECON_TOL = 1e-4


@pytest.fixture(scope="module")
def lc(cuda):
    import laminocam_b200 as lc
    return lc


def problem(lc, n=47, nth=40, seed=3):
    rng = np.random.default_rng(seed)
    th = np.arange(nth) * np.pi / nth
    y = rng.standard_normal((1, nth, n)).astype(np.float32)
    pg = lc.PolarGrid2D(th, n)
    rhs = lc.backproj2d(y, pg, (1, n, n))
    return th, pg, rhs


def test_cg_over_nufft_normal_operator(lc, cuda):
    torch = cuda
    n = 47
    th, pg, rhs = problem(lc, n)
    x = lc.cgsolver_op(lambda v: lc.sysmat2d(v, pg), rhs, torch.zeros_like(rhs), 5, 0.0, 0.0)
    A = lambda v: O.sysmat2d_nufft(v, th, n)
    ref = O.cgsolver(A, rhs.cpu().numpy().astype(np.float64), np.zeros((1, n, n)), 5, 0, 0).x
    assert O.rel_l2(x.cpu().numpy(), ref) < RECON_TOL


def test_split_bregman_over_nufft_normal_operator(lc, cuda):
    torch = cuda
    n = 47
    th, pg, rhs = problem(lc, n, seed=4)
    x = lc.split_bregman_op(lambda v: lc.sysmat2d(v, pg), rhs, torch.zeros_like(rhs), 0.05, 2.0, 4, 2, 0.0, 0.0)
    A = lambda v: O.sysmat2d_nufft(v, th, n)
    ref = O.split_bregman(A, rhs.cpu().numpy().astype(np.float64), np.zeros((1, n, n)), 0.05, 2.0, 4, 2, 0, 0)
    assert O.rel_l2(x.cpu().numpy(), ref) < RECON_TOL


def test_callback_toeplitz_equals_psf_handle_solver(lc, cuda):
    torch = cuda
    n = 63
    th, pg, rhs = problem(lc, n, 60, seed=5)
    psf = lc.PointSpreadFunction2D(pg, n, 1)
    a, ia = lc.cgsolver_op(psf.convolve, rhs, torch.zeros_like(rhs), 8, 0.0, 0.0, return_info=True)
    b, ib = lc.cgsolver(psf, rhs, torch.zeros_like(rhs), 8, 0.0, 0.0, return_info=True)
    assert ia.iters == ib.iters == 8
    assert O.rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-5


def test_failing_callback_stops_the_solve(lc, cuda):
    torch = cuda
    th, pg, rhs = problem(lc)

    def bad(v):
        raise ValueError("operator failed")
    with pytest.raises(ValueError, match="operator failed"):
        lc.cgsolver_op(bad, rhs, torch.zeros_like(rhs), 3, 0.0, 0.0)
    # the context still works afterwards
    x = lc.cgsolver_op(lambda v: lc.sysmat2d(v, pg), rhs, torch.zeros_like(rhs), 2, 0.0, 0.0)
    assert torch.isfinite(x).all()

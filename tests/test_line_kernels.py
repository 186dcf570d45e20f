"""Register-plan line kernels of the Toeplitz apply (the column passes along y
and, in 2D, the fused y pass) against the oracle's FP64 FFT convolution with
the device's own FP64 PSF kernel.

The volume sizes pick padded lengths P = next_smooth(2n - 1) that reach every
kernel variant: even P with a half-length plan (two transforms of P/2, the
Toeplitz case), odd P with a full-length plan, and an even P without a
half-length plan (full-length plan).  The generic shared-memory kernel gives
the same numbers (LC_LINE_KERNELS=0); the tolerance is the one of the
Toeplitz parity tests."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5

# n -> padded P (plan, variant):
#   700 -> 1458 (729 = 9*9*9, two halves)     340 -> 729 (full length)
#   230 ->  486 (243 = 9*9*3, two halves)     115 -> 243 (full length)
#    90 ->  192 ( 96 = 8*4*3, two halves)      45 ->  96 (full length)
SIZES = [700, 340, 230, 115, 90, 45]


@pytest.fixture(scope="module")
def lc(cuda):
    import laminocam_b200 as lc
    return lc


def to_np(t):
    return t.detach().cpu().numpy().astype(np.float64)


def oracle_convolve(psf, x):
    K = psf.kernel()
    if psf.P[0] == 1:
        return O.convolve2d(x, O.PSF2D(psf.P[2], K, np.fft.rfft2(K)))
    return O.convolve3d(x, O.PSF3D(tuple(psf.P), K, np.fft.rfftn(K)))


@pytest.mark.parametrize("n", SIZES)
def test_toeplitz3d_line_kernels(lc, n):
    rng = np.random.default_rng(100 + n)
    nth = 12
    th = np.arange(nth) * 2 * np.pi / nth
    pg = lc.PolarGrid(th, np.full(nth, -np.deg2rad(30.0)), np.zeros(nth), n, n)
    x = rng.random((3, n, n)).astype(np.float32)
    psf = lc.PointSpreadFunction(pg, x.shape)
    assert psf.P[1] == lc.next_fast_dim(2 * n - 1)
    got = to_np(psf.convolve(x))
    want = oracle_convolve(psf, x)
    err = O.rel_l2(got, want)
    assert err < TOL, (n, psf.P, err)


# one slice size per register plan: the half length P/2 of n (P = next_smooth(2n - 1))
# walks 64, 72, 81, 96, 108, 128, ..., 1152, 1296 (every plan of the kernels)
SIZES_2D = [60, 70, 77, 90, 100, 125, 140, 150, 180, 200, 230, 250, 270, 300, 340, 375, 400, 450,
            500, 550, 600, 700, 750, 800, 900, 1000, 1100, 1200, 45, 115]


@pytest.mark.parametrize("n", SIZES_2D)
def test_toeplitz2d_line_kernels(lc, n):
    rng = np.random.default_rng(200 + n)
    nth = 16
    th = np.arange(nth) * np.pi / nth
    pg = lc.PolarGrid2D(th, n)
    ns = 2 if n < 400 else 1
    x = rng.random((ns, n, n)).astype(np.float32)
    psf = lc.PointSpreadFunction2D(pg, n, ns)
    got = to_np(psf.convolve(x))
    want = oracle_convolve(psf, x)
    err = O.rel_l2(got, want)
    assert err < TOL, (n, psf.P, err)

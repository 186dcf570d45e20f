"""Direct z stage of the 3D Toeplitz apply against the oracle.

When the angle set is closed under the mirror that negates kz (every
laminography scan with beta = 0 over a full or half turn), the kernel is even
in z and the z stage of the apply runs as a real symmetric Toeplitz product
per (ky, kx) column instead of the zero-padded FFT, multiply and inverse FFT
(include/toeplitz.h:95-129 is the reference's FFT convolution it replaces).
The depths below reach every compile-time row count of the direct kernel
(4, 8, ..., 32, 40, 48) and one depth above its limit (the FFT form); a scan
over a quarter turn is not mirror-closed and keeps the FFT form.  Parity is
against the oracle's FP64 FFT convolution with the device's own FP64 kernel,
at the tolerance of the other Toeplitz parity tests."""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lc(cuda):
    import laminocam_b200 as lc
    return lc


def grid(lc, nth, n, turn):
    th = np.arange(nth) * turn / nth
    return lc.PolarGrid(th, np.full(nth, -np.deg2rad(30.0)), np.zeros(nth), n, n)


def check(lc, pg, dims, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(dims).astype(np.float32)
    psf = lc.PointSpreadFunction(pg, dims)
    got = psf.convolve(x).detach().cpu().numpy().astype(np.float64)
    K = psf.kernel()
    want = O.convolve3d(x, O.PSF3D(tuple(psf.P), K, np.fft.rfftn(K)))
    return O.rel_l2(got, want)


@pytest.mark.parametrize("n1", [1, 3, 5, 8, 11, 16, 19, 24, 27, 29, 31, 37, 45, 48, 49])
def test_zdirect_depths(lc, n1):
    err = check(lc, grid(lc, 24, 40, 2 * np.pi), (n1, 40, 40), 300 + n1)
    assert err < TOL, (n1, err)


def test_half_turn_mirror(lc):
    # theta in [0, pi): -theta equals pi - theta up to the sign of the row vector
    err = check(lc, grid(lc, 30, 64, np.pi), (29, 64, 64), 7)
    assert err < TOL, err


def test_quarter_turn_fft_form(lc):
    err = check(lc, grid(lc, 20, 48, np.pi / 2), (21, 48, 48), 8)
    assert err < TOL, err


SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import laminocam_b200 as lc
nth, n, n1 = 36, 96, 29
th = np.arange(nth) * 2 * np.pi / nth
pg = lc.PolarGrid(th, np.full(nth, -np.deg2rad(30.0)), np.zeros(nth), n, n)
x = np.random.default_rng(5).standard_normal((n1, n, n)).astype(np.float32)
psf = lc.PointSpreadFunction(pg, x.shape)
y = psf.convolve(x).detach().cpu().numpy()
np.save(sys.argv[2], y)
"""


def test_direct_matches_fft_form(cuda, tmp_path):
    """The same apply with the FFT z stage (LC_ZDIRECT=0) differs only by
    rounding, and the direct form is the one that runs by default."""
    outs = {}
    for flag in ("1", "0"):
        env = dict(os.environ, LC_ZDIRECT=flag)
        path = str(tmp_path / f"y{flag}.npy")
        subprocess.run([sys.executable, "-c", SCRIPT, ROOT, path], env=env, check=True, timeout=600)
        outs[flag] = np.load(path).astype(np.float64)
    d = O.rel_l2(outs["1"], outs["0"])
    assert 0.0 < d < TOL, d

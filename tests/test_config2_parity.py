"""Parity at the laminography benchmark's own size: padded volume [29, 721, 721]
(recon [21, 511, 511]), 360 angles over [0, 2 pi), tilt 30 degrees (gamma =
-30 degrees after the reference's negation), 721 x 721 detector, Toeplitz
grid P = (64, 1458, 1458).  The oracle cannot evaluate whole NUDFTs of 187 M
points, so it checks what it can evaluate exactly at this size:

* 100 random entries of the FP64 PSF kernel against direct sums over all
  187 M lattice points (factored per angle, oracle.lattice_type1_modes);
* the whole Toeplitz apply against the oracle's FP64 FFT convolution with the
  device's FP64 kernel;
* 64 random modes of the backprojection against direct masked sums over all
  points of the detector spectra;
* five Split-Bregman outer iterations (lambda 0.1, mu 10, one CG step each)
  from the device's right-hand side against the oracle's Split-Bregman on the
  FP64 operator.

Tolerances are those of the smaller parity tests: PSF 1e-10, operators 1e-5,
reconstruction 1e-4 relative L2.  The module needs about 12 GB of host memory
and a few minutes of host time.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

NTH = 360
NDET = 721
DIMS = (29, 721, 721)
GAMMA = -np.deg2rad(30.0)


@pytest.fixture(scope="module")
def cfg2(cuda):
    import os

    import laminocam_b200 as lc
    O.set_fft_workers(os.cpu_count() or 1)
    th = np.arange(NTH) * 2 * np.pi / NTH
    pg = lc.PolarGrid(th, np.full(NTH, GAMMA), np.zeros(NTH), NDET, NDET)
    psf = lc.PointSpreadFunction(pg, DIMS)
    assert tuple(psf.P) == (64, 1458, 1458)
    K = psf.kernel()
    yield lc, th, pg, psf, K
    O.set_fft_workers(None)


@pytest.fixture(scope="module")
def oracle_op(cfg2):
    _, _, _, psf, K = cfg2
    return O.PSF3D(tuple(psf.P), K, O._rfftn(K, (0, 1, 2)))


def test_config2_psf_entries_match_direct_sums(cfg2):
    _, th, _, psf, K = cfg2
    rng = np.random.default_rng(2024)
    P = np.array(psf.P)
    # index 0 along an even axis is the unpaired mode -P/2, zeroed on the device
    idx = np.stack([rng.integers(1, p, 100) for p in P], axis=1)
    modes = idx - P // 2
    ref = O.lattice_type1_modes(None, th, np.full(NTH, GAMMA), np.zeros(NTH), NDET, NDET, modes).real
    got = K[idx[:, 0], idx[:, 1], idx[:, 2]]
    err = O.rel_l2(got, ref)
    print(f"config-2 PSF entries: rel L2 {err:.3e}")
    assert err < 1e-10


def test_config2_toeplitz_apply(cfg2, oracle_op):
    _, _, _, psf, _ = cfg2
    rng = np.random.default_rng(2025)
    x = rng.random(DIMS).astype(np.float32)
    got = psf.convolve(x).cpu().numpy().astype(np.float64)
    want = O.convolve3d(x.astype(np.float64), oracle_op)
    err = O.rel_l2(got, want)
    print(f"config-2 Toeplitz apply: rel L2 {err:.3e}")
    assert err < 1e-5


def test_config2_backprojection_modes(cfg2):
    lc, th, pg, _, _ = cfg2
    import scipy.fft
    rng = np.random.default_rng(2026)
    p = rng.random((NTH, NDET, NDET)).astype(np.float32)
    got = lc.backproj(p, pg, DIMS).cpu().numpy().astype(np.float64)
    C = O.fftshift_axis(O.fftshift_axis(p.astype(np.complex128), 1), 2)
    C = scipy.fft.fft2(C, axes=(1, 2), workers=-1, overwrite_x=True)
    C = O.ifftshift_axis(O.ifftshift_axis(C, 1), 2)
    d = np.array(DIMS)
    idx = np.stack([rng.integers(0, n, 64) for n in d], axis=1)
    f = O.lattice_type1_modes(C, th, np.full(NTH, GAMMA), np.zeros(NTH), NDET, NDET, idx - d // 2, mask=True)
    want = f.real / (NDET * NDET)
    err = O.rel_l2(got[idx[:, 0], idx[:, 1], idx[:, 2]], want)
    print(f"config-2 backprojection, 64 modes: rel L2 {err:.3e}")
    assert err < 1e-5


def test_config2_split_bregman_five_outer(cfg2, oracle_op):
    lc, th, pg, psf, _ = cfg2
    import torch
    from laminocam_b200 import synthetic as S
    vol = S.ellipsoid_phantom(DIMS, 40, 1000)
    proj = lc.forward(vol, pg)
    yT = lc.backproj(proj / proj.max(), pg, DIMS)
    x0 = torch.zeros_like(yT)
    got = lc.split_bregman(psf, yT, x0, 0.1, 10.0, 5, 1, 0.0, 0.0).cpu().numpy().astype(np.float64)
    A = lambda v: O.convolve3d(v, oracle_op)
    want = O.split_bregman(A, yT.cpu().numpy().astype(np.float64), np.zeros(DIMS), 0.1, 10.0, 5, 1, 0.0, 0.0)
    err = O.rel_l2(got, want)
    print(f"config-2 Split-Bregman, 5 outer: rel L2 {err:.3e}")
    assert err < 1e-4

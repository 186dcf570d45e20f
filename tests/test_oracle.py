"""CPU tests of the FP64 oracle: golden fixtures, known answers, the reference's
own identities (tests/test_adjoint*.cpp, tests/test_sysmat_toeplitz*.cpp), and
the pin against the reference's sources built with the shim headers."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle import refrun as R

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name))


def test_next_fast_dim_table():
    # include/toeplitz.h:42-51 on the sizes the configs produce
    table = {509: 512, 1441: 1458, 57: 64, 765: 768, 1021: 1024, 4093: 4096, 9: 9, 717: 729,
             41: 48, 1533: 1536, 253: 256, 2045: 2048, 1: 1, 2: 2, 3: 3, 5: 6, 7: 8}
    for n, want in table.items():
        assert O.next_fast_dim(n) == want, n


def test_pad_size_matches_reference_rounding():
    # src/gpu/mbir.cu:46-60: int(n * 1.4142f), forced odd
    assert O.pad_size(511) == 721
    assert O.pad_size(21) == 29
    assert O.pad_size(255) == 359
    assert O.pad_size(383) == 541
    assert O.pad_size(31) == 43
    assert O.pad_size(15) == 21


def test_nudft_single_point_known_answer():
    x = np.array([0.3])
    y = np.array([-1.1])
    F = O.nudft1_2d(np.array([[2.0 + 1j]]), x, y, 5, 4, +1)[0]
    kx = np.arange(-2, 2)
    ky = np.arange(-2, 3)
    want = (2.0 + 1j) * np.exp(1j * (kx[None, :] * 0.3 + ky[:, None] * -1.1))
    assert np.abs(F - want).max() < 1e-13
    c = O.nudft2_2d(want[None], x, y, -1)[0, 0]
    assert abs(c - np.sum(want * np.exp(-1j * (kx[None, :] * 0.3 + ky[:, None] * -1.1)))) < 1e-12


@pytest.mark.parametrize("f", sorted(os.path.basename(p) for p in glob.glob(os.path.join(GOLD, "golden2d_*.npz"))))
def test_oracle_reproduces_golden_2d(f):
    g = load(f)
    th, nr = g["theta"], int(g["nr"])
    vol = g["vol"].astype(np.float64)
    sino = g["sino"].astype(np.float64)
    ns, n = vol.shape[0], vol.shape[1]
    assert O.rel_l2(O.forward2d(vol, th, nr), g["forward2d"]) < 1e-13
    assert O.rel_l2(O.backproj2d(sino, th, (ns, n, n)), g["backproj2d"]) < 1e-13
    psf = O.psf2d(th, nr, n)
    assert O.rel_l2(psf.kernel_hat, g["psf_kernel_hat"]) < 1e-13
    assert O.rel_l2(O.convolve2d(vol, psf), g["toeplitz"]) < 1e-13


@pytest.mark.parametrize("f", ["golden3d_a.npz", "golden3d_b.npz"])
def test_oracle_reproduces_golden_3d(f):
    g = load(f)
    grid = O.Grid3D(g["theta"], g["gamma"], g["beta"], int(g["nrows"]), int(g["ncols"]))
    vol = g["vol"].astype(np.float64)
    proj = g["proj"].astype(np.float64)
    assert O.rel_l2(O.forward3d(vol, grid), g["forward3d"]) < 1e-13
    assert O.rel_l2(O.backproj3d(proj, grid, vol.shape), g["backproj3d"]) < 1e-13
    sh = g["shifts"].astype(np.float64)
    assert O.rel_l2(O.backproj3d(proj, grid, vol.shape, sh), g["backproj3d_shifted"]) < 1e-13


@pytest.mark.parametrize("dims,nang", [((5, 16, 16), 7), ((8, 32, 32), 13)])
def test_adjoint_identity_2d(dims, nang):
    # tests/test_adjoint2d.cpp:56-115 (holds for even detector counts)
    rng = np.random.default_rng(3)
    th = (np.arange(nang) - nang / 2.0) * np.pi / nang
    x = rng.random(dims)
    y = rng.random((dims[0], nang, dims[2]))
    lhs = np.vdot(O.forward2d(x, th), y)
    rhs = np.vdot(x, O.backproj2d(y, th, dims))
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_adjoint_identity_3d():
    rng = np.random.default_rng(4)
    th = (np.arange(7) - 3.5) * np.pi / 7
    grid = O.Grid3D(th, np.full(7, 0.3), np.zeros(7), 16, 16)
    x = rng.random((5, 16, 16))
    y = rng.random((7, 16, 16))
    lhs = np.vdot(O.forward3d(x, grid), y)
    rhs = np.vdot(x, O.backproj3d(y, grid, x.shape))
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


@pytest.mark.parametrize("dims,nang", [((5, 16, 16), 7), ((2, 15, 15), 9)])
def test_toeplitz_equals_nufft_normal_operator_2d(dims, nang):
    # tests/test_sysmat_toeplitz2d.cpp:58-137
    rng = np.random.default_rng(5)
    th = (np.arange(nang) - nang / 2.0) * np.pi / nang
    x = rng.random(dims)
    a = O.sysmat2d_nufft(x, th, dims[2])
    b = O.convolve2d(x, O.psf2d(th, dims[2], dims[2]))
    assert O.rel_l2(b, a) < 1e-12


def test_dirichlet_closed_form_psf_matches_nudft():
    """The closed form used by the CUDA PSF generator: sum_m e^{i u r_m} = sin(pi u)/sin(pi u/n)."""
    rng = np.random.default_rng(6)
    th = np.sort(rng.uniform(0, np.pi, 11))
    nr, n = 13, 9
    P = O.next_fast_dim(2 * n - 1)
    K_exact = O.psf2d(th, nr, n).kernel
    k = np.arange(P) - P // 2
    kx, ky = np.meshgrid(k, k)
    K = np.zeros((P, P))
    for t in th:
        u = kx * np.cos(t) + ky * np.sin(t)
        den = np.sin(np.pi * u / nr)
        with np.errstate(invalid="ignore", divide="ignore"):
            d = np.where(np.abs(den) < 1e-13, nr * np.cos(np.pi * u) / np.cos(np.pi * u / nr),
                         np.sin(np.pi * u) / den)
        K += d
    assert np.abs(K - K_exact).max() / np.abs(K_exact).max() < 1e-12


def _dirichlet(u, n):
    den = np.sin(np.pi * u / n)
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(np.abs(den) < 1e-13, n * np.cos(np.pi * u) / np.cos(np.pi * u / n),
                        np.sin(np.pi * u) / den)


def test_laminography_psf_factorisation_and_table():
    """The tabulated laminography PSF of the CUDA generator, restated in
    numpy: with beta = 0 and one tilt gamma,
        K(k) = D_nx(cg kx - sg ky) * S(sg kx + cg ky, kz),
        S(u, kz) = sum_theta D_ny(cos(theta) u - sin(theta) kz),
    S sampled at spacing 1/32 in u and read back by ten-point Lagrange
    interpolation (weights c_q prod_{m != q} (t - m)).  Against the oracle's
    exact NUDFT kernel (the reference's angle-by-angle sum)."""
    import math
    nth, nr, nc, dims = 40, 29, 31, (5, 30, 30)
    th = -np.pi / 2 + np.arange(nth) * np.pi / nth
    gam = np.deg2rad(-25.0)
    grid = O.Grid3D(th, np.full(nth, gam), np.zeros(nth), nr, nc)
    K_exact = O.psf3d(grid, dims).kernel
    P1, P2, P3 = K_exact.shape
    cg, sg = np.cos(gam), np.sin(gam)
    kz, ky, kx = np.meshgrid(np.arange(P1) - P1 // 2, np.arange(P2) - P2 // 2, np.arange(P3) - P3 // 2,
                             indexing="ij")
    # the table S(u0 + j h, -r), r = |kz|
    h = 1.0 / 32.0
    us = [sg * x + cg * y for x in (-(P3 // 2), P3 - 1 - P3 // 2) for y in (-(P2 // 2), P2 - 1 - P2 // 2)]
    u0 = min(us) - 6 * h
    nu = int(np.ceil((max(us) - u0) / h)) + 8
    uu = u0 + np.arange(nu) * h
    nrz = P1 // 2 + 1
    T = np.zeros((nrz, nu))
    for r in range(nrz):
        for t in th:
            T[r] += _dirichlet(np.cos(t) * uu + np.sin(t) * r, nr)
    # ten-point interpolation
    c = np.array([(-1) ** (9 - q) / (math.factorial(q) * math.factorial(9 - q)) for q in range(10)])
    u, w = sg * kx + cg * ky, cg * kx - sg * ky
    t = (u - u0) / h
    j = np.floor(t).astype(int) - 4
    d = (t - j)[..., None] - np.arange(10)
    pre = np.cumprod(np.concatenate([np.ones(d.shape[:-1] + (1,)), d[..., :-1]], axis=-1), axis=-1)
    suf = np.flip(np.cumprod(np.concatenate([np.ones(d.shape[:-1] + (1,)), np.flip(d, -1)[..., :-1]], axis=-1),
                             axis=-1), -1)
    idx = j[..., None] + np.arange(10)
    vals = T[np.abs(kz)[..., None], idx]
    S = np.sum(c * pre * suf * vals, axis=-1)
    K = _dirichlet(w, nc) * S
    err = np.abs(K - K_exact).max() / np.abs(K_exact).max()
    assert err < 1e-12, err


@pytest.mark.parametrize("three_d", [False, True])
def test_zero_centred_spectrum_is_real_after_dropping_unpaired_planes(three_d):
    """The CUDA PSF keeps Re(FFT(K0)) with K0 the zero-centred kernel whose -P/2
    planes are zeroed: that spectrum is real for any angle set, and the cropped
    convolution with it equals the reference's centred convolution."""
    rng = np.random.default_rng(11)
    if three_d:
        th = np.sort(rng.uniform(0, 2 * np.pi, 5))
        grid = O.Grid3D(th, np.full(5, -0.5), np.full(5, 0.2), 10, 11)
        x = rng.random((4, 8, 9))
        psf = O.psf3d(grid, x.shape)
        K, ref = psf.kernel.copy(), O.convolve3d(x, psf)
    else:
        th = np.sort(rng.uniform(0, np.pi, 7))   # no mirror symmetry
        x = rng.random((1, 12, 12))
        psf = O.psf2d(th, 13, 12)
        K, ref = psf.kernel.copy()[None], O.convolve2d(x, psf)[0][None]
        x = x[0][None]
    for ax, P in enumerate(K.shape):
        if P % 2 == 0 and P > 1:
            sl = [slice(None)] * 3
            sl[ax] = 0
            K[tuple(sl)] = 0
    K0 = np.roll(K, [-(P // 2) for P in K.shape], axis=(0, 1, 2))
    R = np.fft.fftn(K0)
    assert np.abs(R.imag).max() < 1e-12 * np.abs(R.real).max()
    Pd = K.shape
    X = np.zeros(Pd)
    X[:x.shape[0], :x.shape[1], :x.shape[2]] = x
    y = np.fft.irfftn(np.fft.rfftn(X) * R.real[:, :, :Pd[2] // 2 + 1], s=Pd, axes=(0, 1, 2))
    y = y[:x.shape[0], :x.shape[1], :x.shape[2]] / (x.shape[1] * x.shape[2] if three_d else x.shape[2])
    assert O.rel_l2(y, ref) < 1e-12


def test_finite_differences_are_antisymmetric():
    rng = np.random.default_rng(7)
    u = rng.random((4, 5, 6))
    v = [rng.random((4, 5, 6)) for _ in range(3)]
    lhs = sum(np.vdot(g, w) for g, w in zip(O.grad(u), v))
    rhs = -np.vdot(u, O.divergence(v))
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


needs_ref = pytest.mark.skipif(not R.available(), reason="reference build (oracle/_ref) not present")


@needs_ref
def test_pin_oracle_against_reference_sources_2d():
    rng = np.random.default_rng(8)
    th = np.arange(6) * np.pi / 6 + 0.05
    x = rng.random((2, 11, 11))
    y = rng.random((2, 6, 13))
    assert O.rel_l2(O.forward2d(x, th, 13), R.forward2d(x, th, 13)) < 1e-12
    assert O.rel_l2(O.backproj2d(y, th, (2, 11, 11)), R.backproj2d(y, th, 11)) < 1e-12
    P, kh, st, sn = R.psf2d(th, 13, 11, x)
    psf = O.psf2d(th, 13, 11)
    assert P == psf.psf_n
    assert O.rel_l2(psf.kernel_hat, kh) < 1e-12
    assert O.rel_l2(O.convolve2d(x, psf), st) < 1e-12


@needs_ref
def test_pin_finite_differences_against_reference():
    rng = np.random.default_rng(9)
    u = rng.random((4, 6, 7))
    g, d = R.grad(u)
    go = O.grad(u)
    for a in range(3):
        assert O.rel_l2(go[a], g[a]) < 1e-14
    assert O.rel_l2(O.divergence(go), d) < 1e-14
    # the reference CPU stencil is interior-only (src/finitediff.cpp:26-90)
    gc, _ = R.grad(u, cpu_stencil=True)
    oc = O.grad_cpu(u)
    for a in range(3):
        assert O.rel_l2(oc[a], gc[a]) < 1e-14


@needs_ref
def test_pin_split_bregman_against_reference():
    rng = np.random.default_rng(10)
    th = np.arange(8) * np.pi / 8
    sino = rng.random((1, 8, 11))
    a = R.mbir2d(sino, th, 11, "sb", 3, 0.0, 0.0, lam=0.1, mu=5.0, inner=2)
    b = O.mbir2d(sino, th, (1, 11, 11), "sb", 3, 0.0, 0.0, lam=0.1, mu=5.0, inner=2)
    assert O.rel_l2(b, a) < 1e-10


def test_fp32_cg_drifts_from_fp64_cg():
    """Unregularised CG on a noisy ellipse sinogram (n = 63, 60 angles), run by
    the oracle in FP64 and by an FP32 emulation of the same CG on the same
    FP64 operator (only the vectors and the operator outputs are rounded to
    float32).  After 5 iterations the two agree within the 1e-4
    reconstruction bound; after 50 they are more than 1e-2 apart.  The
    normal equations of tomography without density compensation are so
    ill-conditioned that CG amplifies rounding at the 1e-7 level into a
    percent-level difference of the iterate, whatever the code that
    computes it: a long FP32 CG cannot be held to 1e-4 of FP64 CG."""
    from laminocam_b200 import synthetic as S
    n, nth = 63, 60
    th = np.arange(nth) * np.pi / nth
    ph = S.ellipse_phantom(n, 10, 1001)
    sino = O.forward2d(ph[None].astype(np.float64), th, n)
    sino = S.add_noise(sino.astype(np.float32), 0.01, 2001).astype(np.float64)
    sino /= sino.max()
    rhs = O.backproj2d(sino, th, (1, n, n))
    psf = O.psf2d(th, n, n)
    A = lambda v: O.convolve2d(v, psf)
    drift = {}
    for iters in (5, 50):
        ref = O.cgsolver(A, rhs, np.zeros_like(rhs), iters, 0, 0).x
        drift[iters] = O.rel_l2(O.cgsolver_fp32(A, rhs, iters), ref)
    print("FP32 CG drift from FP64 CG:", drift)
    assert drift[5] < 1e-4
    assert drift[50] > 1e-2


@pytest.mark.skipif(not R.bench_available(), reason="oracle/_ref/ref_bench is not built")
def test_timing_build_fft_matches_numpy():
    """The FFTW stand-in of the timing build (multithreaded Stockham / Bluestein)
    against numpy: complex transforms of both signs including non-2^p 3^q
    lengths, and real transforms with even and odd last dimensions."""
    rng = np.random.default_rng(0)
    for shp in [(8,), (9,), (7,), (721,), (3, 5, 4), (16, 24, 18), (5, 7, 11)]:
        a = rng.standard_normal(shp) + 1j * rng.standard_normal(shp)
        for sign in (-1, 1):
            want = np.fft.fftn(a) if sign < 0 else np.fft.ifftn(a) * a.size
            assert O.rel_l2(R.fast_fft("c2c", a, sign), want) < 1e-13, (shp, sign)
    for shp in [(10,), (6, 12), (4, 6, 18), (3, 5, 7), (2, 3, 1458), (2, 729)]:
        a = rng.standard_normal(shp)
        h = np.fft.rfftn(a)
        assert O.rel_l2(R.fast_fft("r2c", a), h) < 1e-13, shp
        want = np.fft.irfftn(h, s=shp, axes=tuple(range(len(shp)))) * a.size
        assert O.rel_l2(R.fast_fft("c2r", h, shape=shp), want) < 1e-13, shp


@pytest.mark.skipif(not R.bench_available(), reason="oracle/_ref/ref_bench is not built")
@pytest.mark.parametrize("tol", [1e-6, 5e-4])
def test_timing_build_nufft_matches_exact_sums(tol):
    """The FINUFFT stand-in of the timing build (ES kernel, colour-scheduled
    spreading) against the exact non-uniform DFTs, type 1 and 2 in 2D and 3D,
    within twice its requested tolerance (FINUFFT's tolerance is an estimate
    of the relative error, not a bound; the reference's float path asks
    5e-4); the 3D type 1 case cuts the fine grid into many y and z blocks."""
    rng = np.random.default_rng(1)
    M = 3000
    x, y, z = (rng.uniform(-np.pi, np.pi, M) for _ in range(3))
    c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    n2, n3 = 12, 17
    assert O.rel_l2(R.fast_nufft(1, 2, (n3, n2), +1, tol, x, y, None, c)[0],
                    O.nudft1_2d(c[None], x, y, n2, n3, +1)[0]) < 2 * tol
    F = rng.standard_normal((n2, n3)) + 1j * rng.standard_normal((n2, n3))
    assert O.rel_l2(R.fast_nufft(2, 2, (n3, n2), -1, tol, x, y, None, F), O.nudft2_2d(F[None], x, y, -1)[0]) < 2 * tol
    n1, n2, n3 = 40, 70, 30
    assert O.rel_l2(R.fast_nufft(1, 3, (n3, n2, n1), +1, tol, x, y, z, c),
                    O.nudft1_3d(c, x, y, z, n1, n2, n3, +1)) < 2 * tol
    F = rng.standard_normal((6, 10, 9)) + 1j * rng.standard_normal((6, 10, 9))
    assert O.rel_l2(R.fast_nufft(2, 3, (9, 10, 6), -1, tol, x, y, z, F), O.nudft2_3d(F, x, y, z, -1)) < 2 * tol

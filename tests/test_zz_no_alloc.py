"""The allocation-free Toeplitz entry point, lc_sysmat2d_toeplitz_noalloc.

It exists for callers that cannot allocate device memory while they run (an
acquisition loop that owns all device memory, a host that forbids cudaMalloc
after start-up because it can synchronise the device).  Its output must equal
the FP64 oracle's Toeplitz apply and the regular lc_sysmat_toeplitz on two
calls in a row (the second call reuses the static arrays the first one left),
and on a third call with another image size (the shared twiddle table is
rewritten for its P); the device's free memory must not change across the
calls; sizes beyond its fixed maximum must be rejected.  The test only calls
through the C ABI; the buffers it passes are allocated by the test before the
free memory is read.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5  # same tolerance as the Toeplitz parity tests


def _noalloc(lib, stream, spec, P, x, y, ns, n):
    return lib.lc_sysmat2d_toeplitz_noalloc(stream, C.c_void_p(spec.data_ptr()), P, C.c_void_p(x.data_ptr()),
                                            C.c_void_p(y.data_ptr()), ns, n)


def test_noalloc_matches_oracle_and_regular_toeplitz(cuda):
    torch = cuda
    import laminocam_b200 as lc
    lib = lc._lib.load()
    rng = np.random.default_rng(77)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream or 1)
    # the set-up call loads the device code (and with it the static arrays)
    assert lib.lc_sysmat2d_toeplitz_noalloc(None, None, 0, None, None, 0, 0) == 0
    cases = []
    for n, nth, ns in ((95, 70, 3), (95, 70, 3), (63, 50, 2)):
        th = np.arange(nth) * np.pi / nth
        psf = lc.PointSpreadFunction2D(lc.PolarGrid2D(th, n), n, ns)
        K = psf.kernel()
        opsf = O.PSF2D(K.shape[0], K, np.fft.rfft2(K))
        spec = torch.as_tensor(psf.spectrum(), device="cuda").contiguous()
        x = torch.as_tensor(rng.random((ns, n, n)).astype(np.float32), device="cuda")
        want = psf.convolve(x)
        y = torch.full_like(x, float("nan"))
        cases.append((n, ns, psf.P[2], opsf, spec, x, want, y))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for n, ns, P, _, spec, x, _, y in cases:
        assert _noalloc(lib, stream, spec, P, x, y, ns, n) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    for call, (n, ns, P, opsf, spec, x, want, y) in enumerate(cases):
        got = y.cpu().numpy().astype(np.float64)
        assert np.isfinite(got).all(), call
        ref = O.convolve2d(x.cpu().numpy().astype(np.float64), opsf)
        assert O.rel_l2(got, ref) < TOL, call
        assert O.rel_l2(got, want.cpu().numpy().astype(np.float64)) < TOL, call


def test_noalloc_rejects_sizes_beyond_its_maximum(cuda):
    torch = cuda
    import laminocam_b200 as lc
    lib = lc._lib.load()
    LC_ERR_TOO_LARGE = 5
    n = 1023
    P = lc.next_fast_dim(2 * n - 1)           # 2048: 1023 x 1025 complex per slice
    ns = 3                                    # 3 slices exceed the 2^21-element scratch
    spec = torch.zeros((P, P // 2 + 1), dtype=torch.float32, device="cuda")
    x = torch.zeros((ns, n, n), dtype=torch.float32, device="cuda")
    y = torch.zeros_like(x)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream or 1)
    assert _noalloc(lib, stream, spec, P, x, y, ns, n) == LC_ERR_TOO_LARGE
    n = 2047                                  # P = 4096 is allowed, but one slice is 2047 x 2049 > 2^21
    P = lc.next_fast_dim(2 * n - 1)
    assert _noalloc(lib, stream, spec, P, x, y, 1, n) == LC_ERR_TOO_LARGE
    assert _noalloc(lib, stream, spec, P + 1, x, y, 1, n) != 0

"""The allocation-free Toeplitz entry point, lc_sysmat2d_toeplitz_noalloc.

It exists for callers that cannot allocate device memory while they run (an
acquisition loop that owns all device memory, a host that forbids cudaMalloc
after start-up).  Its output must equal the regular lc_sysmat_toeplitz on two
calls in a row (the second call reuses the static scratch array left by the
first), and sizes beyond its fixed maximum must be rejected.  The test only
calls through the C ABI; the buffers it passes are allocated by the test.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5  # same tolerance as the Toeplitz parity tests


def test_noalloc_matches_regular_toeplitz_twice(cuda):
    torch = cuda
    import laminocam_b200 as lc
    lib = lc._lib.load()
    rng = np.random.default_rng(77)
    n, nth, ns = 95, 70, 3
    th = np.arange(nth) * np.pi / nth
    pg = lc.PolarGrid2D(th, n)
    psf = lc.PointSpreadFunction2D(pg, n, ns)
    P = psf.P[2]
    spec = torch.as_tensor(psf.spectrum(), device="cuda").contiguous()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream or 1)
    for call in range(2):
        x = torch.as_tensor(rng.random((ns, n, n)).astype(np.float32), device="cuda")
        want = psf.convolve(x)
        y = torch.full_like(x, float("nan"))
        rc = lib.lc_sysmat2d_toeplitz_noalloc(stream, C.c_void_p(spec.data_ptr()), P,
                                              C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), ns, n)
        assert rc == 0, rc
        torch.cuda.synchronize()
        got = y.cpu().numpy().astype(np.float64)
        assert np.isfinite(got).all()
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
    rc = lib.lc_sysmat2d_toeplitz_noalloc(stream, C.c_void_p(spec.data_ptr()), P, C.c_void_p(x.data_ptr()),
                                          C.c_void_p(y.data_ptr()), ns, n)
    assert rc == LC_ERR_TOO_LARGE
    n = 2047                                  # P = 4096 is allowed, but one slice is 2047 x 2049 > 2^21
    P = lc.next_fast_dim(2 * n - 1)
    rc = lib.lc_sysmat2d_toeplitz_noalloc(stream, C.c_void_p(spec.data_ptr()), P, C.c_void_p(x.data_ptr()),
                                          C.c_void_p(y.data_ptr()), 1, n)
    assert rc == LC_ERR_TOO_LARGE
    rc = lib.lc_sysmat2d_toeplitz_noalloc(stream, C.c_void_p(spec.data_ptr()), P + 1, C.c_void_p(x.data_ptr()),
                                          C.c_void_p(y.data_ptr()), 1, n)
    assert rc != 0

"""FP64 CPU oracle for the LaminoCam MBIR hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``laminocam_b200``) may import
this module; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg
of ``bench.py`` use it, and only as the checker.

This is a numpy restatement, in double precision, of the reference's CPU path
(all citations are into the aryabhatt/laminocam sources):

* polar grids            include/polar_grid2d.h:50-65, include/polar_grid.h:52-94,
                         include/rotation.h:28-56
* NUFFT type 1 / type 2  include/nufft.h:37-95 (FINUFFT, iflag +1 / -1, modes in
                         increasing "CMCL" order, dimension 1 = x fastest).  The
                         reference calls FINUFFT at tol 1e-12 in double
                         (include/finufft_plan.h:48); this oracle evaluates the
                         exact non-uniform DFT instead, which is the quantity that
                         FINUFFT approximates, through separable matrix products.
* FFTs                   include/fft.h:76-184 (FFTW: unnormalised, FORWARD = e^{-i})
* fftshift / ifftshift   include/fftutils.h:34-161 (roll by floor(n/2) / ceil(n/2))
* projections            src/projection.cpp:42-182, src/gradient.cpp:32-79
* Toeplitz PSF           include/toeplitz.h:42-129, include/toeplitz2d.h:81-125
* padding / cropping     include/padding.h:34-190
* CG                     src/conjgrad.cpp:33-76 (and src/gpu/conjgrad.cu:45-108)
* Split-Bregman          src/bregman.cpp:36-94 (and src/gpu/bregman.cu:88-165)
* finite differences     src/gpu/finitediff.cu:28-222 (zero-padded central
                         differences; the semantics of the production GPU build)
* orchestration          src/gpu/mbir2d.cu:36-85, src/gpu/mbir.cu:41-167,
                         include/mbir2d_prep.h:44-65

Pinning: the reference ships no golden vectors.  This oracle is pinned against
the reference's own C++ sources compiled unmodified against self-written
FFTW/FINUFFT shim headers (``oracle/ref_build/``), whose direct long-double
DFT and NUDFT sums are restated independently of this module, whenever the
reference sources are available to build them (``LAMINOCAM_REF``).  See
``tests/test_oracle.py``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

PI = math.pi


# ---------------------------------------------------------------------------
# sizes
# ---------------------------------------------------------------------------
def next_fast_dim(n: int) -> int:
    """Smallest 2^p * 3^q >= n (include/toeplitz.h:42-51)."""
    best = 1
    while best < n:
        best <<= 1
    q3 = 3
    while q3 < best:
        x = q3
        while x < n:
            x <<= 1
        if x < best:
            best = x
        q3 *= 3
    return best


def make_odd(n: int) -> int:
    """Even sizes drop by one (include/config.h:377, include/padding.h:40-43)."""
    return n - 1 if n % 2 == 0 else n


def pad_size(n: int, factor: float = 1.4142) -> int:
    """int(n * factor) in float32, forced odd (src/gpu/mbir.cu:46-60)."""
    v = int(np.float32(n) * np.float32(factor))
    return make_odd(v)


# ---------------------------------------------------------------------------
# polar grids
# ---------------------------------------------------------------------------
def polar_grid2d(theta, ncols):
    """x = r cos(theta), y = r sin(theta), r_k = (k+1/2) 2pi/ncols - pi.

    include/polar_grid2d.h:50-65.  Returns arrays of shape (ntheta, ncols).
    """
    theta = np.asarray(theta, dtype=np.float64)
    dr = 2.0 * PI / ncols
    r = (np.arange(ncols) + 0.5) * dr - PI
    x = np.cos(theta)[:, None] * r[None, :]
    y = np.sin(theta)[:, None] * r[None, :]
    return x, y


def rotation_transpose(theta, gamma, beta):
    """transpose(Rx(theta) Ry(beta) Rz(gamma)) (include/rotation.h:28-56)."""
    ct, st = math.cos(theta), math.sin(theta)
    cb, sb = math.cos(beta), math.sin(beta)
    cg, sg = math.cos(gamma), math.sin(gamma)
    return np.array([
        [cb * cg, ct * sg + st * sb * cg, st * sg - ct * sb * cg],
        [-cb * sg, ct * cg - st * sb * sg, st * cg + ct * sb * sg],
        [sb, -st * cb, ct * cb],
    ])


def polar_grid3d(theta, gamma, beta, nrows, ncols):
    """Rotated detector-plane Fourier samples with the |q|<=pi mask.

    include/polar_grid.h:52-94.  Returns x, y, z, w of shape (ntheta, nrows, ncols).
    """
    ntheta = len(theta)
    dX = 2.0 * PI / ncols
    dY = 2.0 * PI / nrows
    qX = (np.arange(ncols) + 0.5) * dX - PI
    qY = (np.arange(nrows) + 0.5) * dY - PI
    x = np.empty((ntheta, nrows, ncols))
    y = np.empty_like(x)
    z = np.empty_like(x)
    for i in range(ntheta):
        R = rotation_transpose(theta[i], gamma[i], beta[i])
        x[i] = R[0, 0] * qX[None, :] + R[0, 1] * qY[:, None]
        y[i] = R[1, 0] * qX[None, :] + R[1, 1] * qY[:, None]
        z[i] = R[2, 0] * qX[None, :] + R[2, 1] * qY[:, None]
    w = ((np.abs(x) <= PI) & (np.abs(y) <= PI) & (np.abs(z) <= PI)).astype(np.float64)
    return x, y, z, w


# ---------------------------------------------------------------------------
# exact non-uniform DFTs (FINUFFT semantics)
# ---------------------------------------------------------------------------
def mode_range(n: int) -> np.ndarray:
    """k in [-floor(n/2), floor((n-1)/2)], increasing (FINUFFT modeord=0)."""
    return np.arange(-(n // 2), (n - 1) // 2 + 1, dtype=np.float64)


_CHUNK = 8192


def nudft1_2d(c, x, y, n2, n3, iflag=+1):
    """Type 1: F[s, ky, kx] = sum_j c[s, j] exp(iflag*i*(kx x_j + ky y_j)).

    c: (ns, M) complex; x, y: (M,).  Output (ns, n2, n3).
    """
    c = np.atleast_2d(np.asarray(c, dtype=np.complex128))
    x = np.ravel(x)
    y = np.ravel(y)
    kx = mode_range(n3)
    ky = mode_range(n2)
    out = np.zeros((c.shape[0], n2, n3), dtype=np.complex128)
    for s0 in range(0, x.size, _CHUNK):
        sl = slice(s0, s0 + _CHUNK)
        Ex = np.exp(iflag * 1j * np.outer(x[sl], kx))   # (m, n3)
        Ey = np.exp(iflag * 1j * np.outer(y[sl], ky))   # (m, n2)
        for s in range(c.shape[0]):
            out[s] += Ey.T @ (c[s, sl][:, None] * Ex)
    return out


def nudft2_2d(F, x, y, iflag=-1):
    """Type 2: c[s, j] = sum_k F[s, ky, kx] exp(iflag*i*(kx x_j + ky y_j))."""
    F = np.asarray(F, dtype=np.complex128)
    if F.ndim == 2:
        F = F[None]
    ns, n2, n3 = F.shape
    x = np.ravel(x)
    y = np.ravel(y)
    kx = mode_range(n3)
    ky = mode_range(n2)
    out = np.zeros((ns, x.size), dtype=np.complex128)
    for s0 in range(0, x.size, _CHUNK):
        sl = slice(s0, s0 + _CHUNK)
        Ex = np.exp(iflag * 1j * np.outer(x[sl], kx))
        Ey = np.exp(iflag * 1j * np.outer(y[sl], ky))
        for s in range(ns):
            out[s, sl] = np.sum((Ey @ F[s]) * Ex, axis=1)
    return out


def nudft1_3d(c, x, y, z, n1, n2, n3, iflag=+1):
    """Type 1 in 3D: F[kz, ky, kx] = sum_j c_j exp(iflag*i*(kx x + ky y + kz z))."""
    c = np.ravel(np.asarray(c, dtype=np.complex128))
    x, y, z = np.ravel(x), np.ravel(y), np.ravel(z)
    kx, ky, kz = mode_range(n3), mode_range(n2), mode_range(n1)
    out = np.zeros((n1, n2, n3), dtype=np.complex128)
    for s0 in range(0, x.size, _CHUNK):
        sl = slice(s0, s0 + _CHUNK)
        Ex = np.exp(iflag * 1j * np.outer(x[sl], kx))
        Ey = np.exp(iflag * 1j * np.outer(y[sl], ky))
        Ez = np.exp(iflag * 1j * np.outer(z[sl], kz))
        cz = c[sl][:, None] * Ez                          # (m, n1)
        for a in range(n1):
            out[a] += Ey.T @ (cz[:, a][:, None] * Ex)
    return out


def nudft2_3d(F, x, y, z, iflag=-1):
    """Type 2 in 3D: c_j = sum_k F[kz, ky, kx] exp(iflag*i*(kx x + ky y + kz z))."""
    F = np.asarray(F, dtype=np.complex128)
    n1, n2, n3 = F.shape
    x, y, z = np.ravel(x), np.ravel(y), np.ravel(z)
    kx, ky, kz = mode_range(n3), mode_range(n2), mode_range(n1)
    out = np.zeros(x.size, dtype=np.complex128)
    for s0 in range(0, x.size, _CHUNK):
        sl = slice(s0, s0 + _CHUNK)
        Ex = np.exp(iflag * 1j * np.outer(x[sl], kx))
        Ey = np.exp(iflag * 1j * np.outer(y[sl], ky))
        Ez = np.exp(iflag * 1j * np.outer(z[sl], kz))
        acc = np.zeros(Ex.shape[0], dtype=np.complex128)
        for a in range(n1):
            acc += Ez[:, a] * np.sum((Ey @ F[a]) * Ex, axis=1)
        out[sl] = acc
    return out


def lattice_type1_modes(C, theta, gamma, beta, nrows, ncols, modes, iflag=+1, mask=False):
    """Selected modes of the 3D type-1 sum over the rotated detector lattices
    of polar_grid3d: f_k = sum_j c_j exp(iflag i k.x_j) for each row (kz, ky,
    kx) of ``modes``, exactly, with c = C (ntheta, nrows, ncols), times the
    |q| <= pi mask when ``mask``.  Per angle the exponent is qX (k.R[:, 0]) +
    qY (k.R[:, 1]), so the lattice sum factors into a matrix product of
    nrows x ncols values with two exponential vectors: O(M K) work for K
    modes, the direct sum at full-size grids."""
    modes = np.asarray(modes, dtype=np.float64).reshape(-1, 3)
    kz, ky, kx = modes[:, 0], modes[:, 1], modes[:, 2]
    qX = (np.arange(ncols) + 0.5) * (2.0 * PI / ncols) - PI
    qY = (np.arange(nrows) + 0.5) * (2.0 * PI / nrows) - PI
    out = np.zeros(modes.shape[0], dtype=np.complex128)
    for i in range(len(theta)):
        R = rotation_transpose(theta[i], gamma[i], beta[i])
        u = kx * R[0, 0] + ky * R[1, 0] + kz * R[2, 0]
        v = kx * R[0, 1] + ky * R[1, 1] + kz * R[2, 1]
        Eb = np.exp(iflag * 1j * np.outer(qX, u))   # (ncols, K)
        Ea = np.exp(iflag * 1j * np.outer(qY, v))   # (nrows, K)
        if C is None and not mask:  # unit weights: the sum factors completely
            out += Ea.sum(axis=0) * Eb.sum(axis=0)
            continue
        Ci = np.ones((nrows, ncols), dtype=np.complex128) if C is None else np.asarray(C[i], dtype=np.complex128)
        if mask:
            x = R[0, 0] * qX[None, :] + R[0, 1] * qY[:, None]
            y = R[1, 0] * qX[None, :] + R[1, 1] * qY[:, None]
            z = R[2, 0] * qX[None, :] + R[2, 1] * qY[:, None]
            Ci = Ci * ((np.abs(x) <= PI) & (np.abs(y) <= PI) & (np.abs(z) <= PI))
        out += np.sum(Ea * (Ci @ Eb), axis=0)
    return out


# ---------------------------------------------------------------------------
# shifts and FFT conventions
# ---------------------------------------------------------------------------
def fftshift_axis(a, axis):
    """out[k] = in[(k + floor(n/2)) % n] (include/fftutils.h:34-52)."""
    n = a.shape[axis]
    return np.roll(a, -(n // 2), axis=axis)


def ifftshift_axis(a, axis):
    """out[k] = in[(k + ceil(n/2)) % n] (include/fftutils.h:95-113)."""
    n = a.shape[axis]
    return np.roll(a, -((n + 1) // 2), axis=axis)


_FFT_WORKERS = None


def set_fft_workers(n):
    """Use scipy.fft with n threads for the Toeplitz FFTs (CPU baseline timing)."""
    global _FFT_WORKERS
    _FFT_WORKERS = n


def _rfftn(a, axes):
    if _FFT_WORKERS:
        import scipy.fft
        return scipy.fft.rfftn(a, axes=axes, workers=_FFT_WORKERS)
    return np.fft.rfftn(a, axes=axes)


def _irfftn(a, s, axes):
    if _FFT_WORKERS:
        import scipy.fft
        return scipy.fft.irfftn(a, s=s, axes=axes, workers=_FFT_WORKERS)
    return np.fft.irfftn(a, s=s, axes=axes)


def fft_fwd(a, axes):
    """FFTW_FORWARD, unnormalised."""
    return np.fft.fftn(a, axes=axes)


def fft_bwd(a, axes):
    """FFTW_BACKWARD, unnormalised."""
    return np.fft.ifftn(a, axes=axes, norm="forward")


# ---------------------------------------------------------------------------
# 2D projections (src/projection.cpp:146-182, src/gradient.cpp:55-79)
# ---------------------------------------------------------------------------
def forward2d(volume, theta, nradial=None):
    """Re(fftshift1(IFFT1(ifftshift1(NUFFT2(vol))))) / nr."""
    vol = np.asarray(volume, dtype=np.float64)
    if vol.ndim == 2:
        vol = vol[None]
    nr = vol.shape[2] if nradial is None else nradial
    x, y = polar_grid2d(theta, nr)
    C = nudft2_2d(vol.astype(np.complex128), x, y, -1).reshape(vol.shape[0], len(theta), nr)
    C = ifftshift_axis(C, 2)
    C = fft_bwd(C, (2,))
    C = fftshift_axis(C, 2)
    return C.real / nr


def backproj2d(sino, theta, recon_dims):
    """Re(NUFFT1(ifftshift1(FFT1(fftshift1(y))))) / nr."""
    y = np.asarray(sino, dtype=np.float64)
    if y.ndim == 2:
        y = y[None]
    ns, nth, nr = y.shape
    n1, n2, n3 = recon_dims
    assert n1 == ns
    x, yy = polar_grid2d(theta, nr)
    C = fftshift_axis(y.astype(np.complex128), 2)
    C = fft_fwd(C, (2,))
    C = ifftshift_axis(C, 2)
    F = nudft1_2d(C.reshape(ns, nth * nr), x, yy, n2, n3, +1)
    return F.real / nr


def sysmat2d_nufft(x, theta, nradial):
    """Direct NUFFT normal operator Re(NUFFT1(NUFFT2(x))) / nr (src/gradient.cpp:55-69)."""
    x = np.asarray(x, dtype=np.float64)
    ns, n2, n3 = x.shape
    gx, gy = polar_grid2d(theta, nradial)
    c = nudft2_2d(x.astype(np.complex128), gx, gy, -1)
    F = nudft1_2d(c, gx, gy, n2, n3, +1)
    return F.real / nradial


# ---------------------------------------------------------------------------
# 2D Toeplitz PSF (include/toeplitz2d.h:81-125)
# ---------------------------------------------------------------------------
@dataclass
class PSF2D:
    psf_n: int
    kernel: np.ndarray       # real PSF on the P x P grid, centre at P/2
    kernel_hat: np.ndarray   # R2C spectrum, (P, P/2+1)


def psf2d(theta, nradial, image_size):
    P = next_fast_dim(2 * image_size - 1)
    gx, gy = polar_grid2d(theta, nradial)
    ones = np.ones((1, gx.size), dtype=np.complex128)
    K = nudft1_2d(ones, gx, gy, P, P, +1)[0].real
    return PSF2D(P, K, np.fft.rfft2(K))


def convolve2d(x, psf: PSF2D):
    x = np.asarray(x, dtype=np.float64)
    if x.ndim == 2:
        x = x[None]
    ns, n2, n3 = x.shape
    P = psf.psf_n
    padded = np.zeros((ns, P, P))
    padded[:, :n2, :n3] = x
    Xh = _rfftn(padded, (1, 2)) * psf.kernel_hat[None]
    res = _irfftn(Xh, (P, P), (1, 2)) * (P * P)   # FFTW C2R is unnormalised
    norm = float(P) * float(P) * float(n3)
    c = P // 2
    return res[:, c:c + n2, c:c + n3] / norm


# ---------------------------------------------------------------------------
# 3D projections (src/projection.cpp:42-131, src/gradient.cpp:32-52)
# ---------------------------------------------------------------------------
@dataclass
class Grid3D:
    theta: np.ndarray
    gamma: np.ndarray
    beta: np.ndarray
    nrows: int
    ncols: int

    def points(self):
        return polar_grid3d(self.theta, self.gamma, self.beta, self.nrows, self.ncols)


def phase_shift2d(C, shifts):
    """C *= exp(-i (qx dx + qy dy)) per projection (include/fft.h:53-74)."""
    ns, n2, n3 = C.shape
    qx = (np.arange(n3) + 0.5) * (2 * PI / n3) - PI
    qy = (np.arange(n2) + 0.5) * (2 * PI / n2) - PI
    out = C.copy()
    for i in range(ns):
        dx, dy = shifts[i]
        ph = qx[None, :] * dx + qy[:, None] * dy
        out[i] *= np.exp(-1j * ph)
    return out


def forward3d(volume, grid: Grid3D):
    """CPU semantics: the mask w is applied (src/projection.cpp:42-64)."""
    vol = np.asarray(volume, dtype=np.float64)
    x, y, z, w = grid.points()
    C = nudft2_3d(vol.astype(np.complex128), x, y, z, -1).reshape(x.shape)
    C = C * w
    C = fftshift_axis(fftshift_axis(C, 1), 2)
    C = fft_bwd(C, (1, 2))
    C = ifftshift_axis(ifftshift_axis(C, 1), 2)
    return C.real / (grid.nrows * grid.ncols)


def backproj3d(proj, grid: Grid3D, recon_dims, shifts=None):
    """src/projection.cpp:69-131: shifts, then mask, then type-1."""
    p = np.asarray(proj, dtype=np.float64)
    x, y, z, w = grid.points()
    C = fftshift_axis(fftshift_axis(p.astype(np.complex128), 1), 2)
    C = fft_fwd(C, (1, 2))
    C = ifftshift_axis(ifftshift_axis(C, 1), 2)
    if shifts is not None:
        C = phase_shift2d(C, shifts)
    C = C * w
    n1, n2, n3 = recon_dims
    F = nudft1_3d(C, x, y, z, n1, n2, n3, +1)
    return F.real / (grid.nrows * grid.ncols)


def sysmat3d_nufft(xv, grid: Grid3D):
    """Re(NUFFT1(NUFFT2(x))) / (nrows*ncols), no mask (src/gradient.cpp:32-45)."""
    xv = np.asarray(xv, dtype=np.float64)
    n1, n2, n3 = xv.shape
    x, y, z, _ = grid.points()
    c = nudft2_3d(xv.astype(np.complex128), x, y, z, -1)
    F = nudft1_3d(c, x, y, z, n1, n2, n3, +1)
    return F.real / (grid.nrows * grid.ncols)


@dataclass
class PSF3D:
    dims: tuple
    kernel: np.ndarray
    kernel_hat: np.ndarray   # (P1, P2, P3/2+1)


def psf3d(grid: Grid3D, recon_dims):
    """Unit weights at every grid point, no mask (include/toeplitz.h:61-93)."""
    P = tuple(next_fast_dim(2 * n - 1) for n in recon_dims)
    x, y, z, _ = grid.points()
    K = nudft1_3d(np.ones(x.size), x, y, z, P[0], P[1], P[2], +1).real
    return PSF3D(P, K, np.fft.rfftn(K))


def convolve3d(xv, psf: PSF3D):
    xv = np.asarray(xv, dtype=np.float64)
    n1, n2, n3 = xv.shape
    P1, P2, P3 = psf.dims
    padded = np.zeros((P1, P2, P3))
    padded[:n1, :n2, :n3] = xv
    res = _irfftn(_rfftn(padded, (0, 1, 2)) * psf.kernel_hat, (P1, P2, P3), (0, 1, 2)) * (P1 * P2 * P3)
    norm = float(P1 * P2 * P3) * float(n2 * n3)
    c1, c2, c3 = P1 // 2, P2 // 2, P3 // 2
    return res[c1:c1 + n1, c2:c2 + n2, c3:c3 + n3] / norm


# ---------------------------------------------------------------------------
# padding (include/padding.h:34-190)
# ---------------------------------------------------------------------------
def pad2d_symmetric(arr, factor=1.4142):
    ns, nr, nc = arr.shape
    n2 = make_odd(int(np.float32(factor) * np.float32(nr)))
    n3 = make_odd(int(np.float32(factor) * np.float32(nc)))
    if factor - 1 < 1e-6:
        return arr.copy()
    out = np.zeros((ns, n2, n3), dtype=arr.dtype)
    d1, d2 = (n2 - nr) // 2, (n3 - nc) // 2
    out[:, d1:d1 + nr, d2:d2 + nc] = arr
    return out


def crop3d_symmetric(arr, new_dims):
    d = [(a - b) // 2 for a, b in zip(arr.shape, new_dims)]
    return arr[d[0]:d[0] + new_dims[0], d[1]:d[1] + new_dims[1], d[2]:d[2] + new_dims[2]].copy()


# ---------------------------------------------------------------------------
# finite differences: zero-padded central differences (src/gpu/finitediff.cu)
# grad returns [d/dn3, d/dn2, d/dn1]; divergence is the matching sum.
# ---------------------------------------------------------------------------
def _cdiff(u, axis):
    up = np.zeros_like(u)
    um = np.zeros_like(u)
    sl_hi = [slice(None)] * 3
    sl_lo = [slice(None)] * 3
    sl_hi[axis] = slice(1, None)
    sl_lo[axis] = slice(None, -1)
    up[tuple(sl_lo)] = u[tuple(sl_hi)]     # u[k+1]
    um[tuple(sl_hi)] = u[tuple(sl_lo)]     # u[k-1]
    return 0.5 * (up - um)


def grad(u):
    return [_cdiff(u, 2), _cdiff(u, 1), _cdiff(u, 0)]


def divergence(du):
    return _cdiff(du[0], 2) + _cdiff(du[1], 1) + _cdiff(du[2], 0)


def laplacian(u):
    return divergence(grad(u))


def grad_cpu(u):
    """Interior-only variant of src/finitediff.cpp:26-90 (faces stay 0), for information."""
    n1, n2, n3 = u.shape
    out = [np.zeros_like(u) for _ in range(3)]
    if n1 < 3 or n2 < 3 or n3 < 3:
        return out
    I = (slice(1, -1),) * 3
    out[0][I] = (u[2:, 1:-1, 1:-1] - u[:-2, 1:-1, 1:-1]) / 2
    out[1][I] = (u[1:-1, 2:, 1:-1] - u[1:-1, :-2, 1:-1]) / 2
    out[2][I] = (u[1:-1, 1:-1, 2:] - u[1:-1, 1:-1, :-2]) / 2
    return out


# ---------------------------------------------------------------------------
# solvers (src/conjgrad.cpp:33-76, src/bregman.cpp:36-94)
# ---------------------------------------------------------------------------
@dataclass
class CGResult:
    x: np.ndarray
    iters: int
    residual: float
    dx: float


def cgsolver(A, y, x0, max_iter, tol, xtol, pap_floor=1e-10, history=None):
    """Unpreconditioned CG.  Stops when |pAp| < pap_floor, residual < tol or dx < xtol."""
    x = np.array(x0, dtype=np.float64, copy=True)
    r = y - A(x)
    y_norm = np.linalg.norm(y)
    p = r.copy()
    rs_old = float(np.vdot(r, r).real)
    it = 0
    res = dxv = float("nan")
    for it in range(max_iter):
        Ap = A(p)
        pAp = float(np.vdot(p, Ap).real)
        if abs(pAp) < pap_floor:
            break
        alpha = rs_old / pAp
        step = alpha * p
        x = x + step
        r = r - alpha * Ap
        rs_new = float(np.vdot(r, r).real)
        p = r + (rs_new / rs_old) * p
        rs_old = rs_new
        res = np.linalg.norm(r) / (y_norm + 1e-8)
        dxv = np.linalg.norm(step) / (np.linalg.norm(x) + 1e-8)
        if history is not None:
            history.append((res, dxv))
        if res < tol or dxv < xtol:
            it += 1
            return CGResult(x, it, res, dxv)
    else:
        it = max_iter
    return CGResult(x, it, res, dxv)


def cgsolver_fp32(A, y, max_iter):
    """The CG of cgsolver (x0 = 0, fixed iteration count) as an FP32 device
    code computes it: vectors and operator outputs rounded to float32, the
    scalars alpha and beta and the dot products in FP64.  A check of how far
    any FP32 CG drifts from FP64 CG on the same operator."""
    f32 = np.float32
    r = np.asarray(y, dtype=f32)
    x = np.zeros_like(r)
    p = r.copy()
    rs_old = float(np.vdot(r.astype(np.float64), r.astype(np.float64)))
    for _ in range(max_iter):
        Ap = np.asarray(A(p.astype(np.float64)), dtype=f32)
        pAp = float(np.vdot(p.astype(np.float64), Ap.astype(np.float64)))
        if pAp == 0.0:
            break
        alpha = rs_old / pAp
        x = (x + f32(alpha) * p).astype(f32)
        r = (r - f32(alpha) * Ap).astype(f32)
        rs_new = float(np.vdot(r.astype(np.float64), r.astype(np.float64)))
        p = (r + f32(rs_new / rs_old) * p).astype(f32)
        rs_old = rs_new
    return x.astype(np.float64)


EPSILON = 1e-8


def split_bregman(A, yT, x0, lam, mu, outer_max, inner_max, tol, xtol, history=None):
    """Isotropic-TV Split-Bregman with zero-padded finite differences."""
    x = np.array(x0, dtype=np.float64, copy=True)
    x_old = x.copy()
    d = [np.zeros_like(x) for _ in range(3)]
    b = [np.zeros_like(x) for _ in range(3)]

    def Ap(u):
        return A(u) - mu * laplacian(u)

    for it in range(outer_max):
        rhs = yT - mu * divergence([d[i] - b[i] for i in range(3)])
        x = cgsolver(Ap, rhs, x, inner_max, tol, xtol).x
        dx = grad(x)
        sk = np.sqrt(sum((dx[i] + b[i]) ** 2 for i in range(3)))
        for i in range(3):
            d[i] = np.maximum(0.0, sk - lam / mu) * ((dx[i] + b[i]) / (sk + EPSILON))
        for i in range(3):
            b[i] = b[i] + dx[i] - d[i]
        nd = np.linalg.norm(x - x_old) / (np.linalg.norm(x_old) + EPSILON)
        if history is not None:
            history.append(nd)
        x_old = x.copy()
        if nd < xtol:
            break
    return x


# ---------------------------------------------------------------------------
# orchestration
# ---------------------------------------------------------------------------
def prepare_sinogram(projs):
    """{ntheta, nrows, ncols} -> /max -> {nrows, ntheta, ncols} (include/mbir2d_prep.h:44-65)."""
    p = np.asarray(projs, dtype=np.float64)
    m = p.max()
    if m > 0:
        p = p / m
    return np.ascontiguousarray(np.transpose(p, (1, 0, 2)))


def mbir2d(sino, theta, recon_dims, method="cg", max_iters=50, tol=1e-5, xtol=1e-5,
           lam=0.1, mu=10.0, inner=1):
    """src/gpu/mbir2d.cu:36-85 on an already prepared sinogram {ns, ntheta, nr}."""
    sino = np.asarray(sino, dtype=np.float64)
    rhs = backproj2d(sino, theta, recon_dims)
    psf = psf2d(theta, sino.shape[2], recon_dims[2])
    A = lambda v: convolve2d(v, psf)
    x0 = np.zeros(recon_dims)
    if method == "cg":
        return cgsolver(A, rhs, x0, max_iters, tol, xtol).x
    return split_bregman(A, rhs, x0, lam, mu, max_iters, inner, tol, xtol)


def mbir3d(projs, theta, gamma, beta, recon_dims, shifts=None, method="cg", max_iters=50,
           tol=1e-5, xtol=1e-5, lam=0.1, mu=10.0, inner=1, pad_factor=1.4142):
    """src/gpu/mbir.cu:41-167 for one dataset: normalise, pad, backproject, PSF, solve, crop."""
    p = np.asarray(projs, dtype=np.float64)
    out_dims = tuple(pad_size(n, pad_factor) for n in recon_dims)
    m = p.max()
    if m > 0:
        p = p / m
    p = pad2d_symmetric(p, pad_factor)
    nth = p.shape[0]
    grid = Grid3D(np.asarray(theta, float), np.full(nth, gamma), np.full(nth, beta),
                  p.shape[1], p.shape[2])
    yT = backproj3d(p, grid, out_dims, shifts)
    psf = psf3d(grid, out_dims)
    A = lambda v: convolve3d(v, psf)
    x0 = np.zeros(out_dims)
    if method == "cg":
        x = cgsolver(A, yT, x0, max_iters, tol, xtol).x
    else:
        x = split_bregman(A, yT, x0, lam, mu, max_iters, inner, tol, xtol)
    return crop3d_symmetric(x, recon_dims)


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))

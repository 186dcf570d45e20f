"""laminocam_b200: the LaminoCam MBIR hot path on one NVIDIA B200.

Python mirror of the reference's operator API (tomocam::forward2d, backproj2d,
sysmat2d, PointSpreadFunction2D, forward, backproj, sysmat, PointSpreadFunction,
opt::cgsolver, opt::split_bregman, gpu::MBIR2D, gpu::MBIR; see
include/projection.h:38-68, include/toeplitz*.h, include/optimize.h:74-91 and
include/gpu/tomocam.h:60-93 of aryabhatt/laminocam).  Every call goes through
the C ABI of liblaminocam_b200.so (include/laminocam.h) to hand-written sm_100a
kernels; torch is used only to own device memory.  There is no CPU fallback:
without the library or a GPU every call raises.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import Job2D, LaminocamError, ReconParamsC, SolverParams, SolverStats

__all__ = [
    "Context", "PolarGrid2D", "PolarGrid", "PointSpreadFunction2D", "PointSpreadFunction",
    "forward2d", "backproj2d", "sysmat2d", "forward", "backproj", "sysmat", "cgsolver",
    "split_bregman", "MBIR2D", "MBIR", "ReconParams", "Dataset", "LaminocamError",
    "next_fast_dim", "make_odd", "pad_size", "Server", "JobResult",
]

DEFAULT_TOL = 1e-6


def next_fast_dim(n: int) -> int:
    """Smallest 2^p 3^q >= n (include/toeplitz.h:42-51)."""
    best = 1
    while best < n:
        best <<= 1
    q3 = 3
    while q3 < best:
        x = q3
        while x < n:
            x <<= 1
        best = min(best, x)
        q3 *= 3
    return best


def make_odd(n: int) -> int:
    return n - 1 if n % 2 == 0 else n


def pad_size(n: int, factor: float = 1.4142) -> int:
    return make_odd(int(np.float32(n) * np.float32(factor)))


def _torch():
    import torch
    return torch


def _check(rc: int, ctx: "Context"):
    if rc != 0:
        msg = _lib.load().lc_last_error(ctx.handle).decode(errors="replace")
        raise LaminocamError(f"laminocam error {rc}: {msg}")


class Context:
    """One device context (lc_context).  Work is ordered on torch's current stream."""

    _default: dict = {}

    def __init__(self, device: int = 0):
        torch = _torch()
        if not torch.cuda.is_available():
            raise LaminocamError("laminocam_b200 needs a CUDA device (no CPU fallback)")
        self.lib = _lib.load()
        self.device = device
        h = C.c_void_p()
        with torch.cuda.device(device):
            rc = self.lib.lc_context_create(device, self._stream_handle(), C.byref(h))
        if rc != 0:
            raise LaminocamError(f"lc_context_create failed ({rc})")
        self.handle = h

    def _stream_handle(self):
        torch = _torch()
        s = torch.cuda.current_stream(self.device).cuda_stream if hasattr(self, "device") else 0
        return C.c_void_p(s if s else 1)  # 1 = cudaStreamLegacy

    def sync_stream(self):
        """Points the context at torch's current stream."""
        _check(self.lib.lc_context_set_stream(self.handle, self._stream_handle()), self)

    @classmethod
    def default(cls, device: Optional[int] = None) -> "Context":
        torch = _torch()
        if device is None:
            device = torch.cuda.current_device() if torch.cuda.is_available() else 0
        if device not in cls._default:
            cls._default[device] = Context(device)
        ctx = cls._default[device]
        ctx.sync_stream()
        return ctx

    def synchronize(self):
        _check(self.lib.lc_context_synchronize(self.handle), self)

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                self.lib.lc_context_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


def _dev(a, dtype=None, device=None):
    """Returns a contiguous float32 CUDA tensor view or copy of a."""
    torch = _torch()
    dtype = dtype or torch.float32
    if isinstance(a, torch.Tensor):
        t = a
        if t.device.type != "cuda":
            t = t.to(device=f"cuda:{device or 0}")
        return t.to(dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=f"cuda:{device or 0}")


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _dptr(arr):
    a = np.ascontiguousarray(arr, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


class PolarGrid2D:
    """cpu/gpu::PolarGrid2D (include/polar_grid2d.h:35-66): theta [rad], ncols radial samples."""

    def __init__(self, theta: Sequence[float], ncols: int, ctx: Optional[Context] = None):
        self.ctx = ctx or Context.default()
        self.theta = np.asarray(theta, dtype=np.float64).copy()
        self.ncols = int(ncols)
        th, p = _dptr(self.theta)
        h = C.c_void_p()
        _check(self.ctx.lib.lc_geometry2d_create(self.ctx.handle, p, len(th), self.ncols, C.byref(h)),
               self.ctx)
        self.handle = h

    def nangles(self):
        return len(self.theta)

    def nradial(self):
        return self.ncols

    def dims(self):
        return (1, len(self.theta), self.ncols)

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                self.ctx.lib.lc_geometry_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class PolarGrid:
    """cpu/gpu::PolarGrid (include/polar_grid.h:34-95) plus per-projection shifts."""

    def __init__(self, theta, gamma, beta, nrows: int, ncols: int, shifts=None,
                 ctx: Optional[Context] = None):
        self.ctx = ctx or Context.default()
        n = len(theta)
        self.theta = np.asarray(theta, dtype=np.float64).copy()
        self.gamma = np.broadcast_to(np.asarray(gamma, dtype=np.float64), (n,)).copy()
        self.beta = np.broadcast_to(np.asarray(beta, dtype=np.float64), (n,)).copy()
        self.nrows, self.ncols = int(nrows), int(ncols)
        self.shifts = None if shifts is None else np.ascontiguousarray(shifts, dtype=np.float32).reshape(n, 2)
        _, pt = _dptr(self.theta)
        _, pg = _dptr(self.gamma)
        _, pb = _dptr(self.beta)
        ps = None if self.shifts is None else self.shifts.ctypes.data_as(C.POINTER(C.c_float))
        h = C.c_void_p()
        _check(self.ctx.lib.lc_geometry3d_create(self.ctx.handle, pt, pg, pb, ps, n, self.nrows,
                                                 self.ncols, C.byref(h)), self.ctx)
        self.handle = h

    def dims(self):
        return (len(self.theta), self.nrows, self.ncols)

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                self.ctx.lib.lc_geometry_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


def _as3(a):
    return a.reshape(1, *a.shape) if a.dim() == 2 else a


def forward2d(volume, pg: PolarGrid2D, tol: float = DEFAULT_TOL):
    """forward2d (src/projection.cpp:146-160): {ns, n2, n3} -> {ns, ntheta, nr}."""
    torch = _torch()
    pg.ctx.sync_stream()
    v = _as3(_dev(volume, device=pg.ctx.device))
    ns, n2, n3 = v.shape
    out = torch.empty((ns, pg.nangles(), pg.ncols), dtype=torch.float32, device=v.device)
    _check(pg.ctx.lib.lc_forward2d(pg.ctx.handle, pg.handle, _ptr(v), ns, n2, n3, _ptr(out), tol), pg.ctx)
    return out


def backproj2d(sino, pg: PolarGrid2D, recon_dims, tol: float = DEFAULT_TOL):
    """backproj2d (src/projection.cpp:168-182): {ns, ntheta, nr} -> recon_dims."""
    torch = _torch()
    pg.ctx.sync_stream()
    s = _as3(_dev(sino, device=pg.ctx.device))
    ns = s.shape[0]
    n1, n2, n3 = recon_dims
    if n1 != ns:
        raise LaminocamError("recon_dims[0] must equal the number of sinogram slices")
    out = torch.empty((ns, n2, n3), dtype=torch.float32, device=s.device)
    _check(pg.ctx.lib.lc_backproj2d(pg.ctx.handle, pg.handle, _ptr(s), ns, n2, n3, _ptr(out), tol), pg.ctx)
    return out


class _PSFBase:
    def __init__(self, ctx, geom, dims, psf_fp32=False):
        self.ctx = ctx
        self.geom = geom
        self.dims_ = tuple(int(d) for d in dims)
        h = C.c_void_p()
        _check(ctx.lib.lc_psf_create_ex(ctx.handle, geom.handle, *self.dims_, 1 if psf_fp32 else 0, C.byref(h)),
               ctx)
        self.handle = h
        P = (C.c_int * 3)()
        ne = C.c_long()
        _check(ctx.lib.lc_psf_info(h, P, C.byref(ne)), ctx)
        self.P = tuple(P)
        self.spectrum_elems = ne.value

    def kernel(self) -> np.ndarray:
        """FP64 PSF on the P grid, mode order (centre at P/2)."""
        shape = (self.P[1], self.P[2]) if self.P[0] == 1 else self.P
        out = np.empty(shape, dtype=np.float64)
        _check(self.ctx.lib.lc_psf_kernel(self.ctx.handle, self.handle,
                                          out.ctypes.data_as(C.POINTER(C.c_double))), self.ctx)
        return out

    def spectrum(self) -> np.ndarray:
        """Real R2C half spectrum {P0, P1, P2/2+1} of the zero-centred PSF (float32)."""
        shape = (self.P[0], self.P[1], self.P[2] // 2 + 1)
        out = np.empty(shape, dtype=np.float32)
        _check(self.ctx.lib.lc_psf_spectrum(self.ctx.handle, self.handle,
                                            out.ctypes.data_as(C.POINTER(C.c_float))), self.ctx)
        return out[0] if self.P[0] == 1 else out

    def convolve(self, x):
        """A^T A x (Toeplitz)."""
        torch = _torch()
        self.ctx.sync_stream()
        v = _dev(x, device=self.ctx.device)
        v3 = _as3(v)
        if tuple(v3.shape) != self.dims_:
            raise LaminocamError(f"convolve: input {tuple(v3.shape)} != PSF dims {self.dims_}")
        out = torch.empty_like(v3)
        _check(self.ctx.lib.lc_sysmat_toeplitz(self.ctx.handle, self.handle, _ptr(v3), _ptr(out)), self.ctx)
        return out.reshape(v.shape)

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                self.ctx.lib.lc_psf_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class PointSpreadFunction2D(_PSFBase):
    """PointSpreadFunction2D (include/toeplitz2d.h:40-126) for nslices slices of image_size^2."""

    def __init__(self, pg: PolarGrid2D, image_size: int, nslices: int = 1, psf_fp32: bool = False):
        """psf_fp32: the kernel from a FP32 NUFFT of ones (the reference GPU's
        construction) instead of the exact FP64 closed form."""
        super().__init__(pg.ctx, pg, (nslices, image_size, image_size), psf_fp32)

    def psf_size(self):
        return self.P[1]


class PointSpreadFunction(_PSFBase):
    """PointSpreadFunction (include/toeplitz.h:35-130) for a volume of recon_dims."""

    def __init__(self, pg: PolarGrid, recon_dims, psf_fp32: bool = False):
        super().__init__(pg.ctx, pg, recon_dims, psf_fp32)


def sysmat2d(x, op, tol: float = DEFAULT_TOL):
    """sysmat2d (src/gradient.cpp:55-79): op is a PolarGrid2D (NUFFT path) or a PSF."""
    if isinstance(op, _PSFBase):
        return op.convolve(x)
    torch = _torch()
    op.ctx.sync_stream()
    v = _as3(_dev(x, device=op.ctx.device))
    ns, n2, n3 = v.shape
    out = torch.empty_like(v)
    _check(op.ctx.lib.lc_sysmat2d_nufft(op.ctx.handle, op.handle, _ptr(v), ns, n2, n3, _ptr(out), tol), op.ctx)
    return out


def forward(volume, pg: PolarGrid, tol: float = DEFAULT_TOL):
    """forward (src/projection.cpp:42-64): {n1, n2, n3} -> {ntheta, nrows, ncols}."""
    torch = _torch()
    pg.ctx.sync_stream()
    v = _dev(volume, device=pg.ctx.device)
    n1, n2, n3 = v.shape
    out = torch.empty(pg.dims(), dtype=torch.float32, device=v.device)
    _check(pg.ctx.lib.lc_forward3d(pg.ctx.handle, pg.handle, _ptr(v), n1, n2, n3, _ptr(out), tol), pg.ctx)
    return out


def backproj(proj, pg: PolarGrid, recon_dims, shifts: bool = False, tol: float = DEFAULT_TOL):
    """backproj (src/projection.cpp:69-131); shifts=True uses the grid's shifts."""
    torch = _torch()
    pg.ctx.sync_stream()
    p = _dev(proj, device=pg.ctx.device)
    n1, n2, n3 = recon_dims
    out = torch.empty((n1, n2, n3), dtype=torch.float32, device=p.device)
    _check(pg.ctx.lib.lc_backproj3d(pg.ctx.handle, pg.handle, _ptr(p), n1, n2, n3, int(bool(shifts)),
                                    _ptr(out), tol), pg.ctx)
    return out


def sysmat(x, op, tol: float = DEFAULT_TOL):
    """sysmat (src/gradient.cpp:32-52): op is a PolarGrid (NUFFT path) or a PSF."""
    if isinstance(op, _PSFBase):
        return op.convolve(x)
    torch = _torch()
    op.ctx.sync_stream()
    v = _dev(x, device=op.ctx.device)
    n1, n2, n3 = v.shape
    out = torch.empty_like(v)
    _check(op.ctx.lib.lc_sysmat3d_nufft(op.ctx.handle, op.handle, _ptr(v), n1, n2, n3, _ptr(out), tol), op.ctx)
    return out


@dataclass
class SolveInfo:
    iters: int
    cg_iters_total: int
    residual: float
    dx: float
    stop_reason: int
    elapsed_ms: float


def _solver_params(max_iters, inner, tol, xtol, lam, mu, fp32_scalars=False, poll_every=8,
                   use_graph=False, residual_refresh=1):
    p = SolverParams()
    _lib.load().lc_solver_params_default(C.byref(p))
    p.max_iters, p.inner_iters = int(max_iters), int(inner)
    p.tol, p.xtol, p.lambda_, p.mu = float(tol), float(xtol), float(lam), float(mu)
    p.fp32_scalars = int(bool(fp32_scalars))
    p.poll_every = int(poll_every)
    p.use_graph = int(bool(use_graph))
    p.residual_refresh = int(residual_refresh)
    return p


def _info(st: SolverStats) -> SolveInfo:
    return SolveInfo(st.iters, st.cg_iters_total, st.residual, st.dx, st.stop_reason, st.elapsed_ms)


def cgsolver(A: _PSFBase, y, x0, max_iter: int, tol: float, xtol: float, fp32_scalars=False,
             return_info=False, use_graph=False):
    """opt::cgsolver (src/conjgrad.cpp:33-76) with the Toeplitz operator A."""
    A.ctx.sync_stream()
    yv = _dev(y, device=A.ctx.device)
    x = _dev(x0, device=A.ctx.device).clone()
    st = SolverStats()
    p = _solver_params(max_iter, 1, tol, xtol, 0.1, 10.0, fp32_scalars, use_graph=use_graph)
    _check(A.ctx.lib.lc_cgsolver(A.ctx.handle, A.handle, _ptr(yv), _ptr(x), C.byref(p), C.byref(st)), A.ctx)
    return (x, _info(st)) if return_info else x


def split_bregman(A: _PSFBase, yT, x0, lam: float, mu: float, outer_max: int, inner_max: int,
                  tol: float, xtol: float, fp32_scalars=False, return_info=False, use_graph=False,
                  residual_refresh=1):
    """opt::split_bregman (src/bregman.cpp:36-94) with the Toeplitz operator A.

    residual_refresh: the operator product A x of each outer iteration's
    warm-started residual is computed exactly every this many outer iterations
    and carried by the CG updates in between (1: every outer iteration)."""
    A.ctx.sync_stream()
    yv = _dev(yT, device=A.ctx.device)
    x = _dev(x0, device=A.ctx.device).clone()
    st = SolverStats()
    p = _solver_params(outer_max, inner_max, tol, xtol, lam, mu, fp32_scalars, use_graph=use_graph,
                       residual_refresh=residual_refresh)
    _check(A.ctx.lib.lc_split_bregman(A.ctx.handle, A.handle, _ptr(yv), _ptr(x), C.byref(p), C.byref(st)),
           A.ctx)
    return (x, _info(st)) if return_info else x


def _operator_callback(ctx, A, shape):
    """Wraps A(x) -> y (torch CUDA tensors of `shape`) as an lc_operator_fn;
    the exception of a failing A is kept and re-raised by the caller."""
    torch = _torch()
    from ._lib import OperatorFn
    err = []

    def fn(user, pin, pout, n, stream):
        try:
            x = _tensor_view(pin, shape, torch)
            y = _tensor_view(pout, shape, torch)
            # 0 and 1 are the legacy default stream (cudaStreamLegacy), 2 the
            # per-thread default stream; torch names the first as its default
            st = torch.cuda.ExternalStream(stream) if (stream or 0) > 2 else torch.cuda.default_stream()
            with torch.cuda.stream(st):
                y.copy_(A(x).reshape(shape))
            return 0
        except Exception as ex:  # reported through the status code
            err.append(ex)
            return 1
    return OperatorFn(fn), err


def _tensor_view(ptr, shape, torch):
    """A torch CUDA float32 tensor over device memory at ptr (not owned)."""
    n = int(np.prod(shape))
    cls = type("Ptr", (), {"__cuda_array_interface__": {"shape": (n,), "typestr": "<f4", "data": (ptr, False),
                                                        "version": 3}})
    return torch.as_tensor(cls(), device="cuda").view(*shape)


def cgsolver_op(A, y, x0, max_iter: int, tol: float, xtol: float, ctx: Optional[Context] = None,
                return_info=False):
    """opt::cgsolver (include/optimize.h:89-91) over any operator A: a callable
    taking and returning torch CUDA tensors shaped like y.  Called once per
    iteration from the solver, with the solver's iteration scalars on the
    device (no graph capture)."""
    ctx = ctx or Context.default()
    ctx.sync_stream()
    yv = _dev(y, device=ctx.device)
    x = _dev(x0, device=ctx.device).clone()
    st = SolverStats()
    p = _solver_params(max_iter, 1, tol, xtol, 0.0, 1.0)
    cb, err = _operator_callback(ctx, A, tuple(yv.shape))
    rc = ctx.lib.lc_cgsolver_op(ctx.handle, cb, None, yv.numel(), _ptr(yv), _ptr(x), C.byref(p), C.byref(st))
    if err:
        raise err[0]
    _check(rc, ctx)
    return (x, _info(st)) if return_info else x


def split_bregman_op(AtA, yT, x0, lam: float, mu: float, outer_max: int, inner_max: int, tol: float,
                     xtol: float, ctx: Optional[Context] = None, return_info=False):
    """opt::split_bregman (include/optimize.h:74-77) over any normal operator
    AtA (a callable on torch CUDA tensors shaped like yT, {n1, n2, n3} or
    {n2, n3}); mu times the negative Laplacian is added by the solver."""
    ctx = ctx or Context.default()
    ctx.sync_stream()
    yv = _dev(yT, device=ctx.device)
    x = _dev(x0, device=ctx.device).clone()
    shape = tuple(yv.shape)
    dims = (C.c_int * 3)(*((1,) * (3 - len(shape)) + shape))
    st = SolverStats()
    p = _solver_params(outer_max, inner_max, tol, xtol, lam, mu)
    cb, err = _operator_callback(ctx, AtA, shape)
    rc = ctx.lib.lc_split_bregman_op(ctx.handle, cb, None, dims, _ptr(yv), _ptr(x), C.byref(p), C.byref(st))
    if err:
        raise err[0]
    _check(rc, ctx)
    return (x, _info(st)) if return_info else x


@dataclass
class ReconParams:
    """ReconParams (include/recon_params.h:45-55)."""
    regularizer: str = "unconstrained"  # or "split_bregman"
    recon_dims: tuple = (0, 0, 0)
    max_iters: int = 100
    inner_iters: int = 1
    lam: float = 0.1
    mu: float = 10.0
    tol: float = 1e-5
    xtol: float = 1e-5
    pad_factor: float = 1.4142
    nufft_tol: float = DEFAULT_TOL
    fp32_scalars: bool = False
    poll_every: int = 8
    use_graph: bool = False
    residual_refresh: int = 1
    psf_fp32: bool = False  # PSF kernel from a FP32 NUFFT of ones (the reference GPU's way)

    def to_c(self) -> ReconParamsC:
        r = ReconParamsC()
        _lib.load().lc_recon_params_default(C.byref(r))
        r.method = 1 if self.regularizer == "split_bregman" else 0
        r.solver = _solver_params(self.max_iters, self.inner_iters, self.tol, self.xtol, self.lam,
                                  self.mu, self.fp32_scalars, self.poll_every, self.use_graph,
                                  self.residual_refresh)
        r.nufft_tol = float(self.nufft_tol)
        r.pad_factor = float(self.pad_factor)
        r.psf_fp32 = 1 if self.psf_fp32 else 0
        return r


@dataclass
class Dataset:
    """Dataset_t (include/recon_params.h:34-40): projs {ntheta, nrows, ncols}, radians."""
    projs: np.ndarray
    angles: np.ndarray
    gamma: float = 0.0
    beta: float = 0.0
    shifts: Optional[np.ndarray] = None


def _fptr(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


def MBIR2D(sinogram, theta, params: ReconParams, ctx: Optional[Context] = None, return_info=False):
    """gpu::MBIR2D (src/gpu/mbir2d.cu:36-85) on a prepared sinogram {ns, ntheta, nr} (host)."""
    ctx = ctx or Context.default()
    s, sp = _fptr(sinogram)
    if s.ndim == 2:
        s = s[None]
        s, sp = _fptr(s)
    ns, nth, nr = s.shape
    _, tp = _dptr(theta)
    rd = (C.c_int * 3)(*[int(d) for d in params.recon_dims])
    out = np.empty(tuple(int(d) for d in params.recon_dims), dtype=np.float32)
    st = SolverStats()
    rp = params.to_c()
    _check(ctx.lib.lc_mbir2d(ctx.handle, sp, ns, nth, nr, tp, rd, C.byref(rp),
                             out.ctypes.data_as(C.POINTER(C.c_float)), C.byref(st)), ctx)
    return (out, _info(st)) if return_info else out


def MBIR2D_batch(jobs, params: ReconParams, ctx: Optional[Context] = None, setup_workers: int = 8,
                 return_info=False):
    """Many independent 2D CG reconstructions batched across jobs
    (lc_mbir2d_batch): jobs is a sequence of (sinogram {ntheta, nr} or
    {1, ntheta, nr}, theta, n).  Every CG stage is one launch over all jobs;
    the result of a job does not depend on the other jobs.  Returns the list
    of {1, n, n} reconstructions (and the per-job SolveInfo)."""
    ctx = ctx or Context.default()
    if params.regularizer != "unconstrained":
        raise LaminocamError("MBIR2D_batch: batched jobs use CG (regularizer 'unconstrained')")
    keep, arr = [], (Job2D * len(jobs))()
    outs = []
    for k, (sino, theta, n) in enumerate(jobs):
        s = np.ascontiguousarray(sino, dtype=np.float32)
        s = s.reshape(s.shape[-2], s.shape[-1])
        th = np.ascontiguousarray(theta, dtype=np.float64)
        o = np.empty((1, int(n), int(n)), dtype=np.float32)
        keep += [s, th]
        outs.append(o)
        arr[k].sinogram = s.ctypes.data_as(C.POINTER(C.c_float))
        arr[k].ntheta, arr[k].nradial = s.shape
        arr[k].theta = th.ctypes.data_as(C.POINTER(C.c_double))
        arr[k].n = int(n)
        arr[k].recon = o.ctypes.data_as(C.POINTER(C.c_float))
    st = (SolverStats * len(jobs))()
    rp = params.to_c()
    _check(ctx.lib.lc_mbir2d_batch(ctx.handle, arr, len(jobs), C.byref(rp), int(setup_workers), st), ctx)
    return (outs, [_info(x) for x in st]) if return_info else outs


def _stack_projs(datasets: Sequence[Dataset]) -> np.ndarray:
    """Projections of all datasets stacked along the angle axis, contiguous
    float32 (one contiguous float32 dataset is passed through without a copy)."""
    if len(datasets) == 1:
        return np.ascontiguousarray(datasets[0].projs, dtype=np.float32)
    return np.ascontiguousarray(np.concatenate(
        [np.asarray(d.projs, dtype=np.float32) for d in datasets], axis=0))


def MBIR(datasets: Sequence[Dataset], params: ReconParams, ctx: Optional[Context] = None,
         return_info=False):
    """gpu::MBIR (src/gpu/mbir.cu:41-167): stacks datasets, normalises, pads, solves, crops."""
    ctx = ctx or Context.default()
    projs = _stack_projs(datasets)
    theta = np.concatenate([np.asarray(d.angles, dtype=np.float64) for d in datasets])
    gamma = np.concatenate([np.full(len(d.angles), d.gamma, dtype=np.float64) for d in datasets])
    beta = np.concatenate([np.full(len(d.angles), d.beta, dtype=np.float64) for d in datasets])
    has_shifts = any(d.shifts is not None for d in datasets)
    sh = None
    if has_shifts:
        sh = np.concatenate([np.zeros((len(d.angles), 2), np.float32) if d.shifts is None
                             else np.asarray(d.shifts, np.float32).reshape(-1, 2) for d in datasets])
    p, pp = _fptr(projs)
    _, tp = _dptr(theta)
    _, gp = _dptr(gamma)
    _, bp = _dptr(beta)
    shp = None
    if sh is not None:
        sh, shp = _fptr(sh)
    rd = (C.c_int * 3)(*[int(d) for d in params.recon_dims])
    out = np.empty(tuple(int(d) for d in params.recon_dims), dtype=np.float32)
    st = SolverStats()
    rp = params.to_c()
    nth, nr, nc = p.shape
    _check(ctx.lib.lc_mbir3d(ctx.handle, pp, nth, nr, nc, tp, gp, bp, shp, rd, C.byref(rp),
                             out.ctypes.data_as(C.POINTER(C.c_float)), C.byref(st)), ctx)
    return (out, _info(st)) if return_info else out


@dataclass
class JobResult:
    """Outcome of one server job: the reconstruction and its timings."""
    recon: np.ndarray
    info: SolveInfo
    queue_ms: float
    run_ms: float
    latency_ms: float
    psf_hit: bool
    worker: int
    device_bytes: float


class Server:
    """Reconstruction server on one GPU (lc_server_* in include/laminocam.h).

    Jobs are gpu::MBIR2D / gpu::MBIR reconstructions with the arguments of
    MBIR2D and MBIR.  They queue in FIFO order, and up to `workers` of them run
    at once when their device footprint fits the HBM budget; while the head of
    the queue waits for memory, up to `backfill` later jobs that fit may start
    ahead of it.  2D jobs run on high-priority streams (`priority_2d`).
    Toeplitz spectra are cached per geometry.  `submit2d` / `submit3d` return
    a job id; `wait` returns a JobResult or raises LaminocamError with the
    job's message.
    """

    def __init__(self, device: int = 0, workers: int = 4, hbm_budget_bytes: float = 0.0,
                 psf_cache_bytes: float = 0.0, psf_cache: bool = True, backfill: int = 16,
                 priority_2d: bool = True):
        self.lib = _lib.load()
        p = _lib.ServerParams()
        self.lib.lc_server_params_default(C.byref(p))
        p.device, p.workers = int(device), int(workers)
        p.hbm_budget_bytes, p.psf_cache_bytes = float(hbm_budget_bytes), float(psf_cache_bytes)
        p.psf_cache = int(bool(psf_cache))
        p.backfill = int(backfill)
        p.priority_2d = int(bool(priority_2d))
        h = C.c_void_p()
        rc = self.lib.lc_server_create(C.byref(p), C.byref(h))
        if rc != 0:
            raise LaminocamError(f"lc_server_create failed with code {rc}")
        self.handle = h
        self._pending = {}

    def _fail(self, rc, what):
        msg = self.lib.lc_server_last_error(self.handle)
        raise LaminocamError(f"{what} failed (code {rc}): {msg.decode() if msg else ''}")

    def submit2d(self, sinogram, theta, params: ReconParams) -> int:
        s = np.ascontiguousarray(sinogram, dtype=np.float32)
        if s.ndim == 2:
            s = np.ascontiguousarray(s[None])
        ns, nth, nr = s.shape
        _, tp = _dptr(theta)
        rd = (C.c_int * 3)(*[int(d) for d in params.recon_dims])
        out = np.empty(tuple(int(d) for d in params.recon_dims), dtype=np.float32)
        rp = params.to_c()
        jid = C.c_longlong()
        rc = self.lib.lc_server_submit2d(self.handle, s.ctypes.data, ns, nth, nr, tp, rd, C.byref(rp),
                                         out.ctypes.data, C.byref(jid))
        if rc != 0:
            self._fail(rc, "submit2d")
        self._pending[jid.value] = (s, out)
        return jid.value

    def submit3d(self, datasets: Sequence[Dataset], params: ReconParams) -> int:
        projs = _stack_projs(datasets)
        theta = np.concatenate([np.asarray(d.angles, dtype=np.float64) for d in datasets])
        gamma = np.concatenate([np.full(len(d.angles), d.gamma, dtype=np.float64) for d in datasets])
        beta = np.concatenate([np.full(len(d.angles), d.beta, dtype=np.float64) for d in datasets])
        sh, shp = None, None
        if any(d.shifts is not None for d in datasets):
            sh = np.ascontiguousarray(np.concatenate(
                [np.zeros((len(d.angles), 2), np.float32) if d.shifts is None
                 else np.asarray(d.shifts, np.float32).reshape(-1, 2) for d in datasets]))
            shp = sh.ctypes.data
        _, tp = _dptr(theta)
        _, gp = _dptr(gamma)
        _, bp = _dptr(beta)
        rd = (C.c_int * 3)(*[int(d) for d in params.recon_dims])
        out = np.empty(tuple(int(d) for d in params.recon_dims), dtype=np.float32)
        rp = params.to_c()
        nth, nr, nc = projs.shape
        jid = C.c_longlong()
        rc = self.lib.lc_server_submit3d(self.handle, projs.ctypes.data, nth, nr, nc, tp, gp, bp, shp,
                                         rd, C.byref(rp), out.ctypes.data, C.byref(jid))
        if rc != 0:
            self._fail(rc, "submit3d")
        self._pending[jid.value] = (projs, out, sh)
        return jid.value

    def wait(self, job: int, timeout_s: float = 0.0) -> JobResult:
        """Blocks until the job ends (timeout_s <= 0: no limit)."""
        st = SolverStats()
        info = _lib.JobInfo()
        rc = self.lib.lc_server_wait(self.handle, int(job), float(timeout_s) * 1e3, C.byref(st),
                                     C.byref(info))
        if rc == 6:
            self._fail(rc, f"wait for job {job}")
        bufs = self._pending.pop(int(job), None)
        if rc != 0:
            raise LaminocamError(f"job {job} failed (code {rc}): {info.error.decode()}")
        return JobResult(bufs[1], _info(st), info.queue_ms, info.run_ms, info.latency_ms,
                         bool(info.psf_hit), info.worker, info.device_bytes)

    def stats(self) -> dict:
        s = _lib.ServerStats()
        rc = self.lib.lc_server_get_stats(self.handle, C.byref(s))
        if rc != 0:
            self._fail(rc, "stats")
        return {name: getattr(s, name) for name, _ in s._fields_}

    def reset_stats(self):
        self.lib.lc_server_reset_stats(self.handle)

    def clear_psf_cache(self):
        """Drops the cached Toeplitz spectra and zeroes the hit / miss counts."""
        rc = self.lib.lc_server_clear_psf_cache(self.handle)
        if rc != 0:
            self._fail(rc, "clear_psf_cache")

    def close(self):
        if getattr(self, "handle", None):
            self.lib.lc_server_destroy(self.handle)
            self.handle = None
            self._pending.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

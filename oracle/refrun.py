"""Runs the reference's own C++ sources (built by oracle/ref_build/Makefile into
oracle/_ref/) on given inputs.  TEST INFRASTRUCTURE ONLY: used to pin the numpy
oracle against the reference's code, and never by the product."""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def driver_path(cpu_stencil: bool = False) -> str:
    return os.path.join(REF_DIR, "ref_driver_cpufd" if cpu_stencil else "ref_driver")


def available(cpu_stencil: bool = False) -> bool:
    return os.path.exists(driver_path(cpu_stencil))


def run(op: str, values, cpu_stencil: bool = False) -> np.ndarray:
    flat = np.concatenate([np.ravel(np.asarray(v, dtype=np.float64)) for v in values])
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.f64")
        fout = os.path.join(td, "out.f64")
        flat.tofile(fin)
        subprocess.run([driver_path(cpu_stencil), op, fin, fout], check=True,
                       env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1)))
        return np.fromfile(fout, dtype=np.float64)


def forward2d(vol, theta, nr):
    ns, n2, n3 = vol.shape
    out = run("forward2d", [[ns, n2, n3, len(theta), nr], theta, vol])
    return out.reshape(ns, len(theta), nr)


def backproj2d(sino, theta, n):
    ns, nth, nr = sino.shape
    out = run("backproj2d", [[ns, nth, nr, n, n], theta, sino])
    return out.reshape(ns, n, n)


def psf2d(theta, nr, n, x):
    """Returns P, kernel_hat (P, P/2+1), Toeplitz sysmat2d(x), NUFFT sysmat2d(x)."""
    ns = x.shape[0]
    out = run("psf2d", [[len(theta), nr, n, ns], theta, x])
    P = int(out[0])
    nh = P * (P // 2 + 1)
    kh = out[1:1 + 2 * nh].view(np.complex128).reshape(P, P // 2 + 1)
    rest = out[1 + 2 * nh:]
    nv = ns * n * n
    return P, kh, rest[:nv].reshape(ns, n, n), rest[nv:2 * nv].reshape(ns, n, n)


def mbir2d(sino, theta, n, method, iters, tol, xtol, lam=0.1, mu=10.0, inner=1):
    ns, nth, nr = sino.shape
    m = 0 if method == "cg" else 1
    out = run("mbir2d", [[ns, nth, nr, n, m, iters, tol, xtol, lam, mu, inner], theta, sino])
    return out.reshape(ns, n, n)


def grad(u, cpu_stencil=False):
    n1, n2, n3 = u.shape
    out = run("grad", [[n1, n2, n3], u], cpu_stencil=cpu_stencil).reshape(4, n1, n2, n3)
    return [out[0], out[1], out[2]], out[3]


def proj3d(vol, proj, theta, gamma, beta, shifts):
    """forward, backproj, backproj(shifts), sysmat(NUFFT), P dims, kernel_hat, sysmat(PSF)."""
    n1, n2, n3 = vol.shape
    nth, nrows, ncols = proj.shape
    out = run("proj3d", [[nth, nrows, ncols, n1, n2, n3], theta, gamma, beta,
                         np.asarray(shifts).ravel(), vol, proj])
    o = 0
    fw = out[o:o + proj.size].reshape(proj.shape); o += proj.size
    bp = out[o:o + vol.size].reshape(vol.shape); o += vol.size
    bps = out[o:o + vol.size].reshape(vol.shape); o += vol.size
    sm = out[o:o + vol.size].reshape(vol.shape); o += vol.size
    P = tuple(int(v) for v in out[o:o + 3]); o += 3
    nk = P[0] * P[1] * (P[2] // 2 + 1)
    kh = out[o:o + 2 * nk].view(np.complex128).reshape(P[0], P[1], P[2] // 2 + 1); o += 2 * nk
    st = out[o:o + vol.size].reshape(vol.shape)
    return dict(forward=fw, backproj=bp, backproj_shifted=bps, sysmat_nufft=sm, P=P,
                kernel_hat=kh, sysmat_toeplitz=st)


def mbir3d(projs, theta, gamma, beta, recon_dims, method, iters, tol, xtol, lam=0.1, mu=10.0,
           inner=1):
    nth, nrows, ncols = projs.shape
    m = 0 if method == "cg" else 1
    out = run("mbir3d", [[nth, nrows, ncols, *recon_dims, m, iters, tol, xtol, lam, mu, inner,
                          gamma, beta], theta, projs])
    return out.reshape(recon_dims)


def bench_path() -> str:
    return os.path.join(REF_DIR, "ref_bench")


def bench_available() -> bool:
    return os.path.exists(bench_path())


def _run_bench(op: str, values) -> np.ndarray:
    flat = np.concatenate([np.ravel(np.asarray(v, dtype=np.float64)) for v in values])
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.f64")
        fout = os.path.join(td, "out.f64")
        flat.tofile(fin)
        subprocess.run([bench_path(), op, fin, fout], check=True,
                       env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1)))
        return np.fromfile(fout, dtype=np.float64)


def fast_fft(kind: str, a, sign: int = -1, double: bool = True, shape=None):
    """The timing build's FFTW stand-in: kind 'c2c' (a complex, any rank),
    'r2c' (a real), 'c2r' (a half spectrum; shape = the real output shape)."""
    a = np.asarray(a)
    k = {"c2c": 0, "r2c": 1, "c2r": 2}[kind]
    dims = list(a.shape) if kind != "c2r" else list(shape)
    data = np.stack([a.real, a.imag], axis=-1).ravel() if np.iscomplexobj(a) or kind != "r2c" else a.ravel()
    out = _run_bench("check_fft", [[k, 1 if double else 0, len(dims)], dims, [sign], data])
    if kind == "c2r":
        return out.reshape(dims)
    if kind == "r2c":
        dims = dims[:-1] + [dims[-1] // 2 + 1]
    return out.view(np.complex128).reshape(dims)


def fast_nufft(nu_type: int, dim: int, modes, iflag: int, tol: float, x, y, z, data, double: bool = True):
    """The timing build's FINUFFT stand-in: type 1 (data = c[M] -> f[modes])
    or type 2 (data = f -> c[M]); modes = (n1, n2, n3), dimension 1 fastest."""
    M = len(x)
    nm = list(modes) + [1] * (3 - len(modes))
    zz = np.zeros(M) if z is None else z
    yy = np.zeros(M) if y is None else y
    d = np.asarray(data, dtype=np.complex128).ravel()
    out = _run_bench("check_nufft", [[nu_type, dim], nm, [iflag, tol, 1 if double else 0, M], x, yy, zz,
                                     np.stack([d.real, d.imag], axis=-1).ravel()])
    out = out.view(np.complex128)
    return out.reshape(nm[2], nm[1], nm[0])[:, :, :] if nu_type == 1 else out


def prec_path() -> str:
    return os.path.join(REF_DIR, "ref_prec")


def prec_available() -> bool:
    return os.path.exists(prec_path())


def _run_prec(op: str, values) -> np.ndarray:
    flat = np.concatenate([np.ravel(np.asarray(v, dtype=np.float64)) for v in values])
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.f64")
        fout = os.path.join(td, "out.f64")
        flat.tofile(fin)
        subprocess.run([prec_path(), op, fin, fout], check=True,
                       env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1)))
        return np.fromfile(fout, dtype=np.float64)


def ref_forward2d(vol, theta, nr, double=True):
    """The reference's forward2d (src/projection.cpp:146-160) in double (FINUFFT
    tol 1e-12) or float (tol 5e-4), on the timing build's FFT/NUFFT stand-ins
    (the zero-padded GPU finite differences)."""
    n = vol.shape[-1]
    out = _run_prec("forward2d" if double else "forward2d_f32", [[n, len(theta), nr], theta, vol])
    return out.reshape(1, len(theta), nr)


def ref_precision2d(sino, theta, n, xprobe, cg_iters, sb_outer, sb_inner, lam, mu, double=True):
    """The reference's backproj2d, sysmat2d(xprobe, PSF), cgsolver and
    split_bregman in double (FINUFFT tol 1e-12) or float (5e-4).  Returns
    (rhs, A^T A xprobe, CG recon, Split-Bregman recon), each {1, n, n}."""
    nth, nr = sino.shape[-2], sino.shape[-1]
    out = _run_prec("precision2d" if double else "precision2d_f32",
                    [[n, nth, nr, cg_iters, sb_outer, sb_inner, lam, mu], theta, sino, xprobe])
    return tuple(out[k * n * n:(k + 1) * n * n].reshape(1, n, n) for k in range(4))

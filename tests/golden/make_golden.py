"""Generates the golden fixtures in tests/golden/ from the FP64 oracle.

Every case is cross-checked against the reference's own C++ sources (built by
oracle/ref_build/Makefile into oracle/_ref/) when that build exists, and the
script refuses to write a fixture that disagrees with it by more than 1e-10.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from oracle import refrun as R  # noqa: E402
from laminocam_b200 import synthetic as S  # noqa: E402


def check(name, a, b, tol=1e-10):
    e = O.rel_l2(a, b)
    print(f"  {name}: oracle vs reference rel {e:.2e}")
    if e > tol:
        raise SystemExit(f"{name}: oracle disagrees with the reference build ({e})")


def case2d(tag, ns, n, nth, nr, seed, theta_kind="ref"):
    rng = np.random.default_rng(seed)
    if theta_kind == "ref":   # tests/test_adjoint2d.cpp:52-57
        theta = (np.arange(nth) - nth / 2.0) * np.pi / nth
    else:                     # uniform over [0, pi)
        theta = np.arange(nth) * np.pi / nth
    vol = rng.random((ns, n, n)).astype(np.float32).astype(np.float64)
    sino = rng.random((ns, nth, nr)).astype(np.float32).astype(np.float64)
    fw = O.forward2d(vol, theta, nr)
    bp = O.backproj2d(sino, theta, (ns, n, n))
    sm = O.sysmat2d_nufft(vol, theta, nr)
    psf = O.psf2d(theta, nr, n)
    tp = O.convolve2d(vol, psf)
    # solver inputs: a consistent phantom sinogram (1% noise) with enough angles
    # for a well-posed system, normalised by its maximum (include/mbir2d_prep.h:61-62)
    nth_s = int(np.ceil(1.6 * n))
    theta_s = np.arange(nth_s) * np.pi / nth_s
    ph = np.stack([S.ellipse_phantom(n, 6, 1000 + seed + i) for i in range(ns)]).astype(np.float64)
    ys = S.add_noise(O.forward2d(ph, theta_s, nr), 0.01, 2000 + seed).astype(np.float64)
    ys = (ys / ys.max()).astype(np.float32).astype(np.float64)
    cg = O.mbir2d(ys, theta_s, (ns, n, n), "cg", 10, 0.0, 0.0)
    sb = O.mbir2d(ys, theta_s, (ns, n, n), "sb", 4, 0.0, 0.0, lam=0.05, mu=2.0, inner=2)
    if R.available():
        check("forward2d", fw, R.forward2d(vol, theta, nr))
        check("backproj2d", bp, R.backproj2d(sino, theta, n))
        P, kh, st, sn = R.psf2d(theta, nr, n, vol)
        check("psf2d.kernel_hat", psf.kernel_hat, kh)
        check("sysmat2d.toeplitz", tp, st)
        check("sysmat2d.nufft", sm, sn)
        check("cg", cg, R.mbir2d(ys, theta_s, n, "cg", 10, 0.0, 0.0), 1e-8)
        check("sb", sb, R.mbir2d(ys, theta_s, n, "sb", 4, 0.0, 0.0, lam=0.05, mu=2.0, inner=2), 1e-8)
    np.savez_compressed(os.path.join(HERE, f"{tag}.npz"), theta=theta, vol=vol.astype(np.float32),
                        sino=sino.astype(np.float32), nr=nr, forward2d=fw, backproj2d=bp,
                        sysmat2d_nufft=sm, psf_kernel=psf.kernel, psf_kernel_hat=psf.kernel_hat,
                        toeplitz=tp, theta_solve=theta_s, sino_solve=ys.astype(np.float32),
                        cg10=cg, sb4=sb)
    print(f"wrote {tag}.npz")


def case3d(tag, vol_dims, nth, nrows, ncols, gamma, beta, seed):
    rng = np.random.default_rng(seed)
    theta = np.arange(nth) * 2 * np.pi / nth
    ga = np.full(nth, gamma)
    be = np.full(nth, beta)
    grid = O.Grid3D(theta, ga, be, nrows, ncols)
    vol = rng.random(vol_dims)
    proj = rng.random((nth, nrows, ncols))
    shifts = rng.normal(scale=1.5, size=(nth, 2))
    vol32 = vol.astype(np.float32).astype(np.float64)
    proj32 = proj.astype(np.float32).astype(np.float64)
    sh32 = shifts.astype(np.float32).astype(np.float64)
    fw = O.forward3d(vol32, grid)
    bp = O.backproj3d(proj32, grid, vol_dims)
    bps = O.backproj3d(proj32, grid, vol_dims, sh32)
    sm = O.sysmat3d_nufft(vol32, grid)
    psf = O.psf3d(grid, vol_dims)
    tp = O.convolve3d(vol32, psf)
    if R.available():
        r = R.proj3d(vol32, proj32, theta, ga, be, sh32)
        check("forward3d", fw, r["forward"])
        check("backproj3d", bp, r["backproj"])
        check("backproj3d.shifts", bps, r["backproj_shifted"])
        check("sysmat3d.nufft", sm, r["sysmat_nufft"])
        check("psf3d.kernel_hat", psf.kernel_hat, r["kernel_hat"])
        check("sysmat3d.toeplitz", tp, r["sysmat_toeplitz"])
    np.savez_compressed(os.path.join(HERE, f"{tag}.npz"), theta=theta, gamma=ga, beta=be,
                        nrows=nrows, ncols=ncols, vol=vol.astype(np.float32),
                        proj=proj.astype(np.float32), shifts=shifts.astype(np.float32),
                        forward3d=fw, backproj3d=bp, backproj3d_shifted=bps, sysmat3d_nufft=sm,
                        psf_kernel=psf.kernel, psf_kernel_hat=psf.kernel_hat, toeplitz=tp)
    print(f"wrote {tag}.npz")


def mbir3d_case(tag, projs_dims, recon_dims, gamma, seed):
    rng = np.random.default_rng(seed)
    nth, nrows, ncols = projs_dims
    theta = np.arange(nth) * 2 * np.pi / nth
    vol = S.ellipsoid_phantom(recon_dims, 6, 3000 + seed).astype(np.float64)
    grid = O.Grid3D(theta, np.full(nth, gamma), np.zeros(nth), nrows, ncols)
    projs = S.add_noise(O.forward3d(vol, grid), 0.01, 4000 + seed)
    p64 = projs.astype(np.float64)
    lam, mu = float(np.float32(0.1)), float(np.float32(10.0))
    cg = O.mbir3d(p64, theta, gamma, 0.0, recon_dims, method="cg", max_iters=6, tol=0, xtol=0)
    sb = O.mbir3d(p64, theta, gamma, 0.0, recon_dims, method="sb", max_iters=3, tol=0, xtol=0,
                  lam=lam, mu=mu, inner=1)
    if R.available():
        check("mbir3d.cg", cg, R.mbir3d(p64, theta, gamma, 0.0, recon_dims, "cg", 6, 0.0, 0.0), 1e-8)
        check("mbir3d.sb", sb, R.mbir3d(p64, theta, gamma, 0.0, recon_dims, "sb", 3, 0.0, 0.0), 1e-8)
    np.savez_compressed(os.path.join(HERE, f"{tag}.npz"), theta=theta, gamma=gamma, projs=projs,
                        recon_dims=np.array(recon_dims), cg6=cg, sb3=sb)
    print(f"wrote {tag}.npz")


if __name__ == "__main__":
    print("reference build available:", R.available())
    case2d("golden2d_odd", ns=2, n=15, nth=9, nr=15, seed=11)
    case2d("golden2d_even", ns=1, n=16, nth=7, nr=16, seed=12)
    case2d("golden2d_nr", ns=1, n=21, nth=12, nr=25, seed=13, theta_kind="uniform")
    case3d("golden3d_a", (5, 8, 9), nth=6, nrows=10, ncols=11, gamma=-0.4, beta=0.1, seed=21)
    case3d("golden3d_b", (3, 12, 12), nth=8, nrows=12, ncols=12, gamma=-np.pi / 6, beta=0.0, seed=22)
    mbir3d_case("golden_mbir3d", (16, 9, 9), (5, 9, 9), -np.pi / 6, seed=31)

"""The C++ adapter include/tomocam_b200_adapter.h: the reference's API
(gpu::MBIR2D, forward2d, backproj2d, the PSF convolve, opt::cgsolver over an
opt::Function) over the B200 C ABI.  oracle/ref_build compiles a check
program against the reference's own headers (array.h, recon_params.h,
optimize.h) into oracle/_ref/adapter_check; on the CPU the test checks that it
was built, on the GPU that it computes what the Python API and the FP64
oracle compute."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "adapter_check")


def test_adapter_compiles_against_reference_headers():
    if not os.path.isdir(os.environ.get("LAMINOCAM_REF", "/root/reference")) and not os.path.exists(EXE):
        pytest.skip("no reference headers to compile against, and no prebuilt check program")
    if not os.path.exists(EXE):
        r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle", "ref_build"),
                            f"REF={os.environ.get('LAMINOCAM_REF', '/root/reference')}",
                            os.path.join("..", "_ref", "adapter_check")], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-2000:]
    assert os.access(EXE, os.X_OK)


@pytest.mark.gpu
def test_adapter_runs_the_reference_api_on_the_gpu(cuda):
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/adapter_check is not built")
    import laminocam_b200 as lc
    rng = np.random.default_rng(12)
    n, nth = 63, 60
    th = (np.arange(nth) * np.pi / nth).astype(np.float32).astype(np.float64)
    sino = rng.random((1, nth, n)).astype(np.float32)
    vol = rng.random((1, n, n)).astype(np.float32)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.f64"), os.path.join(td, "out.f64")
        np.concatenate([[n, nth], th, sino.ravel(), vol.ravel()]).astype(np.float64).tofile(fin)
        subprocess.run([EXE, fin, fout], check=True, timeout=300)
        out = np.fromfile(fout, dtype=np.float64)
    k = n * n
    fw = out[:nth * n].reshape(1, nth, n)
    bp, ax, rec, cg = (out[nth * n + i * k: nth * n + (i + 1) * k].reshape(1, n, n) for i in range(4))
    pg = lc.PolarGrid2D(th, n)
    # the same C-ABI calls as the Python API: the same bits
    assert np.array_equal(fw.astype(np.float32), lc.forward2d(vol, pg).cpu().numpy())
    assert np.array_equal(bp.astype(np.float32), lc.backproj2d(sino, pg, (1, n, n)).cpu().numpy())
    psf = lc.PointSpreadFunction2D(pg, n, 1)
    assert np.array_equal(ax.astype(np.float32), psf.convolve(vol).cpu().numpy())
    x = lc.MBIR2D(sino, th, lc.ReconParams(recon_dims=(1, n, n), max_iters=5, tol=0, xtol=0))
    assert np.array_equal(rec.astype(np.float32), x)
    # and the FP64 oracle
    s64 = sino.astype(np.float64)
    assert O.rel_l2(rec, O.mbir2d(s64, th, (1, n, n), "cg", 5, 0.0, 0.0)) < 1e-4
    A = lambda v: O.sysmat2d_nufft(v, th, n)
    ref = O.cgsolver(A, O.backproj2d(s64, th, (1, n, n)), np.zeros((1, n, n)), 5, 0, 0).x
    assert O.rel_l2(cg, ref) < 1e-4

"""Cross-job batching (lc_mbir2d_batch): uneven 2D CG jobs in lockstep, every
stage one launch over the whole batch.

A job's arithmetic does not depend on the rest of the batch (its FFT lines,
its chunking and the order of its reductions are fixed by its own size), so a
job's result is bit-for-bit the same alone and in any mix; with graphs and
without; and with per-job tolerances, each job stops where it stops alone.
Against the FP64 oracle the batch holds the 1e-4 reconstruction bound at
CG(5), like the one-job path (long unregularised CG runs drift in any FP32
CG, see tests/test_oracle.py)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

RECON_TOL = 1e-4


@pytest.fixture(scope="module")
def lc(cuda):
    import laminocam_b200 as lc
    return lc


def job(lc, n, nth, seed):
    from laminocam_b200.synthetic import add_noise, ellipse_phantom
    th = np.arange(nth) * np.pi / nth
    s = lc.forward2d(ellipse_phantom(n, 8, seed)[None], lc.PolarGrid2D(th, n)).cpu().numpy()
    s = add_noise(s, 0.01, seed + 1000)
    return (np.ascontiguousarray(s / s.max(), dtype=np.float32), th, n)


def params(lc, iters, graph=True, tol=0.0):
    return lc.ReconParams(regularizer="unconstrained", recon_dims=(1, 1, 1), max_iters=iters, tol=tol,
                          xtol=0.0, use_graph=graph)


@pytest.fixture(scope="module")
def mix(lc):
    # sizes whose Toeplitz grids (128 ... 2048) use different FFT plans and
    # lines per CTA in one launch
    # (n = 365 has the odd grid P = 729, whose real rows are not packed)
    shapes = [(63, 60), (95, 150), (127, 90), (255, 200), (191, 333), (511, 120), (1023, 90), (63, 61),
              (365, 100)]
    return [job(lc, n, nth, 50 + k) for k, (n, nth) in enumerate(shapes)]


def test_batch_equals_each_job_alone(lc, mix):
    both = lc.MBIR2D_batch(mix, params(lc, 50))
    for j, x in zip(mix, both):
        alone = lc.MBIR2D_batch([j], params(lc, 50))[0]
        assert np.array_equal(x, alone)
        assert np.isfinite(x).all()


def test_batch_graph_equals_eager(lc, mix):
    a = lc.MBIR2D_batch(mix[:4], params(lc, 20, graph=True))
    b = lc.MBIR2D_batch(mix[:4], params(lc, 20, graph=False))
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_batch_matches_oracle_and_single_job_path(lc, mix):
    sel = mix[:3] + mix[-1:]
    out = lc.MBIR2D_batch(sel, params(lc, 5))
    for (s, th, n), x in zip(sel, out):
        ref = O.mbir2d(s.astype(np.float64), th, (1, n, n), "cg", 5, 0.0, 0.0)
        assert O.rel_l2(x, ref) < RECON_TOL
        single = lc.MBIR2D(s, th, lc.ReconParams(recon_dims=(1, n, n), max_iters=5, tol=0, xtol=0))
        assert O.rel_l2(x, single) < RECON_TOL


def test_batch_jobs_stop_on_their_own_tests(lc, mix):
    """With a residual tolerance each job stops at its own iteration; the
    stats report it, and the result equals the job run alone."""
    outs, info = lc.MBIR2D_batch(mix[:5], params(lc, 200, tol=0.05), return_info=True)
    its = [i.iters for i in info]
    assert all(i.stop_reason == 1 and i.iters < 200 for i in info), its
    for j, x, i in zip(mix[:5], outs, info):
        a, ai = lc.MBIR2D_batch([j], params(lc, 200, tol=0.05), return_info=True)
        assert ai[0].iters == i.iters
        assert np.array_equal(a[0], x)


def test_batch_rejects_bad_jobs(lc, mix):
    with pytest.raises(lc.LaminocamError):
        lc.MBIR2D_batch(mix[:2], lc.ReconParams(regularizer="split_bregman", recon_dims=(1, 1, 1)))

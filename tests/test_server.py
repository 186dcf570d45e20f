"""The reconstruction server (lc_server_*) and CUDA-graph replay of the solvers.

Every result the server computes, alone or among concurrent jobs, equals what
the one-job drivers (lc_mbir2d / lc_mbir3d) return for the same arguments bit
for bit: the backprojection sums in exact fixed point, the PSF and the
Toeplitz passes are fixed arithmetic per element, and the solver's reductions
are fixed-order, so neither the other jobs on the device nor a cached PSF
change a result.  The CG cases run 50 iterations, the configuration's count.
Graph replay of the solvers equals eager launches bit for bit; a failing job
must leave the other jobs and the server intact.  Every wait has a time limit,
so a stuck job fails the test instead of stalling the run.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

RECON_TOL = 1e-4
WAIT_S = 300.0


@pytest.fixture(scope="module")
def lc(cuda):
    import laminocam_b200 as lc
    return lc


def sino2d(lc, n, nth, seed):
    from laminocam_b200.synthetic import add_noise, ellipse_phantom
    th = np.arange(nth) * np.pi / nth
    img = ellipse_phantom(n, 8, seed)
    s = lc.forward2d(img[None], lc.PolarGrid2D(th, n)).cpu().numpy()
    s = add_noise(s, 0.01, seed + 1000)
    return (s / s.max()).astype(np.float32), th


def lamino(lc, dims, nth, gamma_deg, seed):
    from laminocam_b200.synthetic import add_noise, ellipsoid_phantom
    th = np.arange(nth) * 2 * np.pi / nth
    vol = ellipsoid_phantom(dims, 6, seed)
    n = dims[1]
    g = -np.deg2rad(gamma_deg)
    pg = lc.PolarGrid(th, np.full(nth, g), np.zeros(nth), n, n)
    p = lc.forward(vol, pg).cpu().numpy()
    p = add_noise(p, 0.01, seed + 1000)
    return p.astype(np.float32), th, g


def params2d(lc, n, method, iters, graph=False):
    return lc.ReconParams(regularizer=method, recon_dims=(1, n, n), max_iters=iters, tol=0.0,
                          xtol=0.0, use_graph=graph)


def test_graph_replay_matches_eager(lc):
    """Same operator and right-hand side: the replayed iterations run the same
    kernels with the same deterministic reductions, so the results agree bit
    for bit."""
    import torch
    n, nth = 95, 90
    th = np.arange(nth) * np.pi / nth
    pg = lc.PolarGrid2D(th, n)
    A = lc.PointSpreadFunction2D(pg, n, 1)
    rng = np.random.default_rng(5)
    y = torch.as_tensor(rng.standard_normal((1, n, n)).astype(np.float32), device="cuda")
    x0 = torch.zeros_like(y)
    a, ia = lc.cgsolver(A, y, x0, 12, 0.0, 0.0, return_info=True)
    b, ib = lc.cgsolver(A, y, x0, 12, 0.0, 0.0, return_info=True, use_graph=True)
    assert ia.iters == ib.iters == 12
    assert torch.equal(a, b)
    a = lc.split_bregman(A, y, x0, 0.1, 10.0, 5, 2, 0.0, 0.0)
    b = lc.split_bregman(A, y, x0, 0.1, 10.0, 5, 2, 0.0, 0.0, use_graph=True)
    assert torch.equal(a, b)


def test_graph_replay_through_the_driver(lc):
    """MBIR2D with graphs against MBIR2D without: the same bits."""
    s, th = sino2d(lc, 95, 90, 11)
    for method, iters in (("unconstrained", 50), ("split_bregman", 5)):
        a = lc.MBIR2D(s, th, params2d(lc, 95, method, iters, graph=False))
        b, info = lc.MBIR2D(s, th, params2d(lc, 95, method, iters, graph=True), return_info=True)
        assert info.iters == iters
        assert np.array_equal(b, a)


def test_graph_replay_with_tolerance_stop(lc):
    """A residual test that fires inside a replayed chunk: the later iterations
    of the chunk are no-ops on the device, so the result and the iteration
    count equal the eager run's."""
    import torch
    n, nth = 63, 60
    th = np.arange(nth) * np.pi / nth
    A = lc.PointSpreadFunction2D(lc.PolarGrid2D(th, n), n, 1)
    rng = np.random.default_rng(6)
    # a right-hand side in the range of the operator, so that CG converges
    xt = torch.as_tensor(rng.standard_normal((1, n, n)).astype(np.float32), device="cuda")
    y = A.convolve(xt)
    x0 = torch.zeros_like(y)
    a, ia = lc.cgsolver(A, y, x0, 200, 1e-2, 0.0, return_info=True)
    b, ib = lc.cgsolver(A, y, x0, 200, 1e-2, 0.0, return_info=True, use_graph=True)
    assert ia.stop_reason == ib.stop_reason == 1
    assert ia.iters == ib.iters < 200
    assert torch.equal(a, b)


def test_server_results_match_single_jobs(lc):
    jobs2d = [(63, 60, 1, "unconstrained", 50), (95, 120, 2, "split_bregman", 4),
              (127, 90, 3, "unconstrained", 50), (63, 60, 4, "split_bregman", 3)]
    data = [sino2d(lc, n, nth, seed) for n, nth, seed, _, _ in jobs2d]
    ref = [lc.MBIR2D(s, th, params2d(lc, n, m, it))
           for (n, _, _, m, it), (s, th) in zip(jobs2d, data)]
    p3, th3, g3 = lamino(lc, (7, 31, 31), 40, 30.0, 5)
    rp3 = lc.ReconParams(regularizer="split_bregman", recon_dims=(7, 31, 31), max_iters=3, tol=0,
                         xtol=0)
    ds = [lc.Dataset(p3, th3, g3, 0.0)]
    ref3 = lc.MBIR(ds, rp3)
    with lc.Server(workers=3) as sv:
        ids = []
        for rep in range(2):  # the second round finds every PSF in the cache
            for (n, _, _, m, it), (s, th) in zip(jobs2d, data):
                ids.append(sv.submit2d(s, th, params2d(lc, n, m, it, graph=rep == 1)))
            ids.append(sv.submit3d(ds, rp3))
        res = [sv.wait(j, WAIT_S) for j in ids]
        st = sv.stats()
    for r, e in zip(res, (ref + [ref3]) * 2):
        assert np.array_equal(r.recon, e)
    assert st["completed"] == len(ids) and st["failed"] == 0
    assert st["psf_hits"] >= 5 and all(r.psf_hit for r in res[5:])
    assert st["p99_ms"] >= st["p50_ms"] > 0


def test_server_result_matches_oracle(lc):
    s, th = sino2d(lc, 63, 60, 21)
    with lc.Server(workers=2) as sv:
        r = sv.wait(sv.submit2d(s, th, params2d(lc, 63, "unconstrained", 5)), WAIT_S)
    xo = O.mbir2d(s.astype(np.float64), th, (1, 63, 63), method="cg", max_iters=5, tol=0, xtol=0)
    assert O.rel_l2(r.recon, xo) < RECON_TOL


def test_server_psf_cache_clear(lc):
    """Clearing the cache drops the spectra and zeroes the counts: the next job
    of a cached geometry builds its PSF again, with the same result."""
    s, th = sino2d(lc, 63, 60, 31)
    prm = params2d(lc, 63, "split_bregman", 3)
    with lc.Server(workers=1) as sv:
        a = sv.wait(sv.submit2d(s, th, prm), WAIT_S)
        b = sv.wait(sv.submit2d(s, th, prm), WAIT_S)
        assert not a.psf_hit and b.psf_hit
        sv.clear_psf_cache()
        st = sv.stats()
        assert st["psf_hits"] == st["psf_misses"] == st["psf_cache_entries"] == 0
        c = sv.wait(sv.submit2d(s, th, prm), WAIT_S)
        assert not c.psf_hit
        assert sv.stats()["psf_misses"] == 1
    assert np.array_equal(c.recon, a.recon)


def test_server_many_workers_uneven_jobs(lc):
    """48 workers on 48 slices of different sizes and angle counts.  The PSF
    and spreading kernels take job-dependent shared memory and launch from
    many threads at once; every job must succeed and equal its one-job run."""
    rng = np.random.default_rng(77)
    jobs = []
    for k in range(48):
        n = int(rng.choice([63, 95, 127]))
        nth = int(rng.integers(90, 721))
        s, th = sino2d(lc, n, nth, 500 + k)
        jobs.append((s, th, n))
    with lc.Server(workers=48) as sv:
        ids = [sv.submit2d(s, th, params2d(lc, n, "split_bregman", 3)) for s, th, n in jobs]
        res = [sv.wait(j, WAIT_S) for j in ids]
        st = sv.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 0
    for (s, th, n), r in list(zip(jobs, res))[:6]:
        ref = lc.MBIR2D(s, th, params2d(lc, n, "split_bregman", 3))
        assert np.array_equal(r.recon, ref)


def test_server_isolates_failing_job(lc):
    s, th = sino2d(lc, 63, 60, 31)
    good = params2d(lc, 63, "unconstrained", 50)
    bad = lc.ReconParams(regularizer="unconstrained", recon_dims=(2, 63, 63), max_iters=4)
    ref = lc.MBIR2D(s, th, good)
    with lc.Server(workers=2) as sv:
        a = sv.submit2d(s, th, good)
        b = sv.submit2d(s, th, bad)  # recon_dims[0] != number of slices: fails when it runs
        c = sv.submit2d(s, th, good)
        ra = sv.wait(a, WAIT_S)
        with pytest.raises(lc.LaminocamError, match="recon_dims"):
            sv.wait(b, WAIT_S)
        rc = sv.wait(c, WAIT_S)
        st = sv.stats()
        rd = sv.wait(sv.submit2d(s, th, good), WAIT_S)  # still serving after the failure
    for r in (ra, rc, rd):
        assert np.array_equal(r.recon, ref)
    assert st["failed"] == 1 and st["completed"] == 2


def test_server_rejects_job_over_budget(lc):
    s, th = sino2d(lc, 63, 60, 41)
    with lc.Server(workers=1, hbm_budget_bytes=1 << 20) as sv:
        with pytest.raises(lc.LaminocamError, match="code 5"):
            sv.submit2d(s, th, params2d(lc, 63, "unconstrained", 3))


def test_server_admission_respects_budget(lc):
    """With a budget for two jobs, no more than two run at once."""
    s, th = sino2d(lc, 127, 90, 51)
    p = params2d(lc, 127, "split_bregman", 3)
    with lc.Server(workers=1) as probe:
        one = probe.wait(probe.submit2d(s, th, p), WAIT_S).device_bytes
    with lc.Server(workers=4, hbm_budget_bytes=2.5 * one) as sv:
        ids = [sv.submit2d(s, th, p) for _ in range(6)]
        res = [sv.wait(j, WAIT_S) for j in ids]
        st = sv.stats()
    assert st["peak_admitted_bytes"] <= 2.5 * one
    assert 1 <= st["peak_running"] <= 2
    for r in res[1:]:
        assert np.array_equal(r.recon, res[0].recon)


def test_server_backfill_starts_small_jobs_ahead_of_a_waiting_head(lc):
    """Budget for one large job: while the second large job waits at the head
    of the queue for memory, small jobs behind it start on the free workers
    (backfill) instead of waiting; with backfill 0 the order is strict FIFO.
    Results are the same either way."""
    # (the footprint estimate holds a fixed 64 MiB per job, so the large job
    # must be large for two small ones to fit beside it)
    sb, thb = sino2d(lc, 1023, 90, 61)
    ss, ths = sino2d(lc, 63, 60, 62)
    big = params2d(lc, 1023, "unconstrained", 50)
    small = params2d(lc, 63, "unconstrained", 50)
    with lc.Server(workers=1) as probe:
        one = probe.wait(probe.submit2d(sb, thb, big), WAIT_S).device_bytes
        ref_small = probe.wait(probe.submit2d(ss, ths, small), WAIT_S).recon
    for backfill in (16, 0):
        with lc.Server(workers=4, hbm_budget_bytes=1.5 * one, backfill=backfill) as sv:
            ids = [sv.submit2d(sb, thb, big), sv.submit2d(sb, thb, big)]
            ids += [sv.submit2d(ss, ths, small) for _ in range(4)]
            res = [sv.wait(j, WAIT_S) for j in ids]
            st = sv.stats()
        assert st["completed"] == 6 and st["failed"] == 0
        for r in res[2:]:
            assert np.array_equal(r.recon, ref_small)
        if backfill:
            assert st["backfilled"] >= 1
            # the small jobs did not wait for the second large job to finish
            assert max(r.queue_ms for r in res[2:]) < res[1].queue_ms + res[1].run_ms
        else:
            assert st["backfilled"] == 0
        assert st["p50_2d_ms"] > 0 and st["p99_2d_ms"] >= st["p50_2d_ms"] and st["p50_3d_ms"] == 0

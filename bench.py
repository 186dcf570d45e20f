#!/usr/bin/env python
"""Benchmark: laminography MBIR reconstructions per second on one B200.

Workload (the reference's laminography configuration): recon_dims [21, 511, 511]
(padded to [29, 721, 721] inside the solver), 40 seeded random ellipsoids,
360 projections over [0, 360 deg), tilt gamma = 30 deg (TOML key, negated
internally like include/config.h:206), 511 x 511 detector, 1% Gaussian noise,
Split-Bregman TV with lambda = 0.1, mu = 10, inner_iters = 1, 100 outer
iterations (tol = 1e-5, xtol = 0 so that every step does the same work), NUFFT
tolerance 1e-6.

A step is one complete reconstruction: normalisation and padding of the
projections, geometry and bin sort, backprojection (type-1 NUFFT), FP64 PSF
generation (no cache), 100 Split-Bregman outer iterations (the first one eager,
the other 99 replayed as a CUDA graph) and the final crop.
`value` is measured with the projections resident in HBM (lc_mbir3d_device);
`e2e` through the host-buffer API (lc_mbir3d) with a pinned host copy in and
the reconstruction copied back out every step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (the path does not shard across GPUs; the
reference's multi-GPU slice streaming has no single-volume exchange), launched
with torch.distributed.run; rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

RECON_DIMS = (21, 511, 511)
NANGLES = 360
DET = (511, 511)
GAMMA_DEG = 30.0
N_ELLIPSOIDS = 40
OUTER = 100
LAM, MU = 0.1, 10.0
NOISE = 0.01
METRIC = "laminography MBIR reconstructions/s (Split-Bregman TV, 100 outer iterations)"
CONFIG = {
    "workload": "laminography Split-Bregman: recon_dims [21,511,511] (padded [29,721,721]), "
                "360 angles over [0,360), tilt 30 deg, 511x511 detector, 40 ellipsoids, 1% noise, "
                "lambda 0.1, mu 10, inner 1, outer 100, NUFFT tol 1e-6",
    "recon_dims": list(RECON_DIMS), "padded_dims": [29, 721, 721], "angles": NANGLES,
    "detector": list(DET), "outer_iters": OUTER, "inner_iters": 1, "lambda": LAM, "mu": MU,
    "tol": 1e-5, "xtol": 0.0, "nufft_tol": 1e-6,
    "l2_policy": "inputs larger than L2 (projections 376 MB, fine grids >1 GB)",
}


def geometry():
    theta = np.arange(NANGLES) * 2 * np.pi / NANGLES
    gamma = -GAMMA_DEG * np.pi / 180.0
    return theta, gamma


def make_projections(lc):
    """Seeded phantom, forward-projected on the GPU (like the reference's
    forward_scalar tool, src/radon.cpp), plus 1% noise."""
    import torch
    from laminocam_b200 import synthetic as S
    theta, gamma = geometry()
    vol = S.ellipsoid_phantom(RECON_DIMS, N_ELLIPSOIDS, 1000)
    pg = lc.PolarGrid(theta, np.full(NANGLES, gamma), np.zeros(NANGLES), DET[0], DET[1])
    proj = lc.forward(torch.as_tensor(vol, device="cuda"), pg)
    proj = proj + NOISE * proj.max() * torch.randn(proj.shape, device="cuda",
                                                   generator=torch.Generator("cuda").manual_seed(2000))
    torch.cuda.synchronize()
    del pg
    return vol, proj.contiguous()


class ClockSampler:
    """Samples the SM clock and the clock-event (throttle) reasons during the
    timed region (every `interval` seconds): read-only NVML queries in this
    process, or nvidia-smi when NVML cannot be loaded."""

    REASONS = [("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap")]

    def __init__(self, index: int, interval: float = 1.0):
        self.index = index
        self.interval = interval
        self.samples = []  # (sm_mhz, sm_max_mhz, [active reasons])
        self.source = None
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)
        # NVML is initialised here, before the timed region: nvmlInit on a
        # host with several GPUs takes long enough to disturb a timed step
        self._nvml_state = None
        try:
            import pynvml as N
            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByIndex(self.index)
            mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
            get = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons",
                          getattr(N, "nvmlDeviceGetCurrentClocksThrottleReasons", None))
            masks = [(name, getattr(N, attr, 0)) for name, attr in self.REASONS]
            self._nvml_state = (N, h, mx, get, masks)
        except Exception:
            self._nvml_state = None

    def _nvml(self):
        if self._nvml_state is None:
            raise RuntimeError("NVML unavailable")
        N, h, mx, get, masks = self._nvml_state
        self.source = "nvml"
        while not self._stop.is_set():
            sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
            bits = get(h) if get else 0
            self.samples.append((float(sm), float(mx), [n for n, m in masks if m and bits & m]))
            self._stop.wait(self.interval)

    def _smi(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        self.source = "nvidia-smi"
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                v = [x.strip() for x in out.split(",")]
                if len(v) >= 6:
                    act = [self.REASONS[i][0] for i in range(4) if v[2 + i].lower() == "active"]
                    self.samples.append((float(v[0]), float(v[1]), act))
            except Exception:
                pass
            self._stop.wait(self.interval)

    def _run(self):
        try:
            self._nvml()
        except Exception:
            self._smi()

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock samples"]}
        sm = [s[0] for s in self.samples]
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(s[1] for s in self.samples),
                "reasons": sorted({r for s in self.samples for r in s[2]}),
                "samples": len(self.samples), "source": self.source}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


REF_BENCH = os.path.join(ROOT, "oracle", "_ref", "ref_bench")


def reference_cpu_run(warmup: int, steps: int, full: bool = False):
    """The reference's own CPU path on this workload, timed on the host cores:
    its sources (src/projection.cpp, gradient.cpp, conjgrad.cpp, bregman.cpp,
    finitediff.cpp, mbir.cpp, include/toeplitz.h) compiled unmodified in float
    against self-written multithreaded FFTW / FINUFFT stand-ins
    (oracle/ref_build, target ref_bench; FINUFFT at the reference's float
    tolerance 5e-4, include/finufft_plan.h:71).  The projections are the
    reference's own forward() of the same seeded phantom plus 1% noise.
    Returns the setup time (the calls of tomocam::MBIR before its solver:
    normalisation, padding, polar grid, backprojection, PSF), the times of
    `steps` single Split-Bregman outer iterations after `warmup` untimed ones,
    and, with `full`, one complete tomocam::MBIR of 100 outer iterations."""
    import tempfile
    from laminocam_b200 import synthetic as S
    if not os.path.exists(REF_BENCH):
        raise RuntimeError("oracle/_ref/ref_bench is not built (needs the reference sources at build time)")
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        ph = os.path.join(td, "phantom.f32")
        S.ellipsoid_phantom(RECON_DIMS, N_ELLIPSOIDS, 1000).astype(np.float32).tofile(ph)
        cmd = [REF_BENCH, "lamino", ph, *map(str, RECON_DIMS), str(NANGLES), str(GAMMA_DEG), str(warmup),
               str(steps)] + (["full"] if full else [])
        out = subprocess.run(cmd, capture_output=True, text=True, check=True,
                             env=dict(os.environ, OMP_NUM_THREADS=str(cores))).stdout
    rec = [json.loads(line) for line in out.splitlines() if line.startswith("{")]
    setup = next(r for r in rec if r["phase"] == "setup")
    outer = [r["seconds"] for r in rec if r["phase"] == "outer"]
    fullr = next((r["seconds"] for r in rec if r["phase"] == "full"), None)
    recon_s = setup["seconds"] + OUTER * float(np.mean(outer))
    return {"cores": cores, "setup_s": setup["seconds"], "backproj_s": setup["backproj_s"],
            "psf_s": setup["psf_s"], "outer_s": outer, "recon_s": recon_s, "full_s": fullr}


def cpu_baseline():
    """Bounded sample of the reference's CPU path (setup and two outer
    iterations, about a minute of host time), scaled to one reconstruction."""
    r = reference_cpu_run(0, 2)
    return {"value": 1.0 / r["recon_s"], "unit": "recons/s", "cores": r["cores"], "kind": "reference",
            "sample": f"the reference's own sources (float, FINUFFT tol 5e-4) on self-written "
                      f"multithreaded FFTW/FINUFFT stand-ins, {r['cores']} OpenMP threads: setup "
                      f"(backprojection + PSF) {r['setup_s']:.1f} s measured once, 2 Split-Bregman outer "
                      f"iterations at {np.mean(r['outer_s']):.2f} s each; one reconstruction = setup + "
                      f"100 outer iterations = {r['recon_s']:.1f} s",
            "setup_s": r["setup_s"], "outer_s": float(np.mean(r["outer_s"]))}


# ncu dram__bytes_read.sum + dram__bytes_write.sum of one Toeplitz apply at the
# padded workload volume [29, 721, 721] (--kernel-case toeplitz): x rows 60 + 62 MB,
# y forward 122 + 190, direct z stage 370 + 189, y inverse 247 + 96, x inverse
# 122 + 32 (writes still in L2 when a pass ends are not counted)
TOEPLITZ_APPLY_DRAM_BYTES = 1492e6

# padded detector of the workload (511 -> int(511 * 1.4142) forced odd)
PADDED_DET = (721, 721)
# conflict-free 32-bit shared-memory reductions per clock per SM (B200, probe)
SHARED_RED_PER_CLK_SM = 30.9

MIX_JOBS = 64
MIX_ITERS = 50


def mix_jobs(lc, count=MIX_JOBS, seed=3000):
    """Uneven 2D slices: n = odd(round(exp(U[ln 128, ln 1024]))), ntheta ~ U{90..720}
    over [0, pi), 10 ellipses each, forward-projected on the GPU, 1% noise,
    normalised by the maximum."""
    import torch
    from laminocam_b200 import synthetic as S
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(count):
        n = int(round(np.exp(rng.uniform(np.log(128), np.log(1024)))))
        n -= (n % 2 == 0)
        nth = int(rng.integers(90, 721))
        th = np.arange(nth) * np.pi / nth
        img = S.ellipse_phantom(n, 10, 1000 + k)
        s = lc.forward2d(torch.as_tensor(img[None], device="cuda"), lc.PolarGrid2D(th, n))
        s = S.add_noise(s.cpu().numpy(), NOISE, 2000 + k)
        jobs.append((np.ascontiguousarray(s / s.max(), dtype=np.float32), th, n))
    torch.cuda.synchronize()
    return jobs


def serving_mix(lc, workers=32):
    """The same 64 uneven 2D CG jobs (50 iterations each) solved (a) one at a time
    the plain way -- float scalars, a host check of the solver state after every
    iteration, no graphs, a PSF built per job -- and (b) submitted together to
    the server: concurrent jobs on 32 streams, CUDA-graph iterations, FP64
    scalars, geometry-keyed PSF cache.  Wall-clock times, host buffers in and
    out.  The error of both forms against the FP64 oracle is measured on one
    small job (n = 63, 60 angles) of the same kind."""
    from oracle import oracle as O
    jobs = mix_jobs(lc)

    def prm(n, plain, iters=MIX_ITERS):
        # plain: tol 1e-30 keeps the per-iteration host check without ever stopping
        return lc.ReconParams(regularizer="unconstrained", recon_dims=(1, n, n), max_iters=iters,
                              tol=1e-30 if plain else 0.0, xtol=0.0, fp32_scalars=plain,
                              poll_every=1 if plain else 8, use_graph=not plain)

    # untimed pass over every job shape (one CG iteration each): fills the FFT
    # launch-tuner cache that both forms share, so neither pays for tuning
    for s, th, n in jobs:
        lc.MBIR2D(s, th, prm(n, True, 1))
    t0 = time.perf_counter()
    plain_out, plain_ms = [], []
    for s, th, n in jobs:
        a = time.perf_counter()
        plain_out.append(lc.MBIR2D(s, th, prm(n, True)))
        plain_ms.append((time.perf_counter() - a) * 1e3)
    t_plain = time.perf_counter() - t0

    with lc.Server(workers=workers) as sv:
        small = min(jobs, key=lambda j: j[2])
        sv.wait(sv.submit2d(small[0], small[1], prm(small[2], False)), 600)
        sv.reset_stats()
        t0 = time.perf_counter()
        ids = [sv.submit2d(s, th, prm(n, False)) for s, th, n in jobs]
        res = [sv.wait(j, 600) for j in ids]
        t_served = time.perf_counter() - t0
        st = sv.stats()
        # the FP64 oracle on one small job of the same kind
        from laminocam_b200 import synthetic as S
        th1 = np.arange(60) * np.pi / 60
        s1 = lc.forward2d(S.ellipse_phantom(63, 10, 4000)[None], lc.PolarGrid2D(th1, 63)).cpu().numpy()
        s1 = np.ascontiguousarray(S.add_noise(s1, NOISE, 4001), dtype=np.float32)
        s1 /= s1.max()
        x_served = sv.wait(sv.submit2d(s1, th1, prm(63, False)), 600).recon
    x_plain = lc.MBIR2D(s1, th1, prm(63, True))
    # (c) cross-job batching: all 64 jobs in lockstep, every CG stage one
    # launch over the batch (lc_mbir2d_batch); setup on 8 worker streams
    bprm = prm(0, False)
    # untimed pass over every job shape (one iteration), as for the other two
    # forms: loads the batched kernels of every plan length and creates the 8
    # setup worker contexts (kept in the caller's context, as the server keeps
    # its workers)
    lc.MBIR2D_batch(jobs, prm(0, False, 1))
    t0 = time.perf_counter()
    bat = lc.MBIR2D_batch(jobs, bprm)
    t_batch = time.perf_counter() - t0
    x_batch = lc.MBIR2D_batch([(s1, th1, 63)], bprm)[0]
    xo = O.mbir2d(s1.astype(np.float64), th1, (1, 63, 63), method="cg", max_iters=MIX_ITERS, tol=0,
                  xtol=0)
    sizes = [j[2] for j in jobs]
    return {
        "workload": f"{MIX_JOBS} uneven 2D slices, n odd log-uniform in [127, 1023], ntheta U{{90..720}} "
                    f"over [0,180), 10 ellipses, 1% noise, CG {MIX_ITERS} iterations (fixed count)",
        "n_range": [min(sizes), max(sizes)],
        "plain": {"recons_per_s": MIX_JOBS / t_plain, "seconds": t_plain,
                  "job_ms_p50": float(np.percentile(plain_ms, 50)),
                  "job_ms_p99": float(np.percentile(plain_ms, 99)),
                  "form": "one job at a time, float scalars, host check every iteration, no graphs, "
                          "PSF built per job"},
        "served": {"recons_per_s": MIX_JOBS / t_served, "seconds": t_served,
                   "latency_ms_p50": st["p50_ms"], "latency_ms_p99": st["p99_ms"],
                   "workers": workers, "peak_running": st["peak_running"],
                   "psf_hits": st["psf_hits"], "psf_misses": st["psf_misses"],
                   "form": "all 64 submitted at once; concurrent streams, CUDA-graph CG iterations, "
                           "FP64 scalars, geometry-keyed PSF cache"},
        "batched": {"recons_per_s": MIX_JOBS / t_batch, "seconds": t_batch,
                    "form": "lockstep batches: each CG stage one launch over every job of a batch "
                            "(6 launches per iteration, 8-iteration CUDA graphs), per-job FP64 "
                            "scalars; setup on 8 worker streams, the larger half iterating while "
                            "the rest is set up"},
        "speedup": t_plain / t_served,
        "speedup_batched": t_plain / t_batch,
        "max_rel_l2_served_vs_plain": max(O.rel_l2(r.recon, p) for r, p in zip(res, plain_out)),
        "max_rel_l2_batched_vs_served": max(O.rel_l2(b, r.recon) for b, r in zip(bat, res)),
        "rel_l2_vs_fp64_oracle_n63": {"served": O.rel_l2(x_served, xo), "plain": O.rel_l2(x_plain, xo),
                                      "batched": O.rel_l2(x_batch, xo)},
        "timing": "wall clock, host buffers in and out",
    }


# config-4 precision study: one large slice, three precisions of the same path
PREC_N, PREC_ANGLES, PREC_ELLIPSES, PREC_NOISE = 2047, 1800, 60, 0.005
PREC_CG, PREC_SB_OUTER, PREC_SB_INNER, PREC_LAM, PREC_MU = 200, 30, 2, 0.05, 10.0


def precision_study(lc, n=PREC_N, nth=PREC_ANGLES, cg_iters=PREC_CG, sb_outer=PREC_SB_OUTER,
                    sb_inner=PREC_SB_INNER):
    """One n x n ellipse slice (60 ellipses), nth angles over [0, 180), 0.5 %
    noise, CG(200) and Split-Bregman (lambda 0.05, mu 10, 30 outer x 2 inner),
    computed three ways and compared with the FP64 oracle (the reference's own
    double path: its sources on the timing build's stand-ins at FINUFFT tol
    1e-12, oracle/_ref/ref_prec):
      default   this build: FP32 spreading, FFTs and vectors, FP64 PSF kernel
                and FP64 CG scalars and reductions
      all_fp32  this build with the PSF kernel from a FP32 NUFFT of ones (the
                reference GPU's construction) and FP32 CG scalars and dots
                (the reference GPU's float accumulation, src/gpu/array_ops.cu:210-213)
      reference_float  the reference's own float CPU path (FINUFFT tol 5e-4,
                include/finufft_plan.h:71), for context
    Relative L2 errors of the projection (noise free), the backprojection of
    the noisy sinogram, A^T A of the phantom, and the two reconstructions."""
    import torch
    from laminocam_b200 import synthetic as S
    from oracle import oracle as O
    from oracle import refrun as R
    th = np.arange(nth) * np.pi / nth
    ph = S.ellipse_phantom(n, PREC_ELLIPSES, 1000)[None].astype(np.float64)
    xprobe = ph / ph.max()
    p64 = R.ref_forward2d(ph, th, n)
    sino = S.add_noise(p64.astype(np.float32), PREC_NOISE, 2000)
    sino = np.ascontiguousarray(sino / sino.max(), dtype=np.float32)
    s64 = sino.astype(np.float64)
    ref = R.ref_precision2d(s64, th, n, xprobe, cg_iters, sb_outer, sb_inner, PREC_LAM, PREC_MU)
    ref32 = R.ref_precision2d(s64, th, n, xprobe, cg_iters, sb_outer, sb_inner, PREC_LAM, PREC_MU, double=False)
    p32ref = R.ref_forward2d(ph, th, n, double=False)
    names = ("backprojection", "AtA", "recon_cg", "recon_sb")
    out = {"workload": f"{n}x{n} slice, {PREC_ELLIPSES} ellipses, {nth} angles over [0,180), "
                       f"{PREC_NOISE * 100:.1f}% noise; CG {cg_iters} iterations; Split-Bregman "
                       f"lambda {PREC_LAM}, mu {PREC_MU}, {sb_outer} outer x {sb_inner} inner",
           "oracle": "the reference's double path (FINUFFT tol 1e-12) on the timing build's stand-ins"}
    out["reference_float"] = {"projection": O.rel_l2(p32ref, p64),
                              **{k: O.rel_l2(a, b) for k, a, b in zip(names, ref32, ref)}}
    pg = lc.PolarGrid2D(th, n)
    proj = lc.forward2d(ph.astype(np.float32), pg).cpu().numpy().astype(np.float64)
    bp = lc.backproj2d(sino, pg, (1, n, n)).cpu().numpy().astype(np.float64)
    for variant, f32 in (("default", False), ("all_fp32", True)):
        psf = lc.PointSpreadFunction2D(pg, n, 1, psf_fp32=f32)
        ax = psf.convolve(xprobe.astype(np.float32)).cpu().numpy().astype(np.float64)
        del psf
        cg = lc.MBIR2D(sino, th, lc.ReconParams(recon_dims=(1, n, n), max_iters=cg_iters, tol=0, xtol=0,
                                               fp32_scalars=f32, psf_fp32=f32, use_graph=True))
        sb = lc.MBIR2D(sino, th, lc.ReconParams(regularizer="split_bregman", recon_dims=(1, n, n),
                                               max_iters=sb_outer, inner_iters=sb_inner, lam=PREC_LAM, mu=PREC_MU,
                                               tol=0, xtol=0, fp32_scalars=f32, psf_fp32=f32, use_graph=True))
        out[variant] = {"projection": O.rel_l2(proj, p64), "backprojection": O.rel_l2(bp, ref[0]),
                        "AtA": O.rel_l2(ax, ref[1]), "recon_cg": O.rel_l2(cg, ref[2]),
                        "recon_sb": O.rel_l2(sb, ref[3])}
    torch.cuda.synchronize()
    return out


STREAM_RATES = (5.0, 20.0, 80.0)
STREAM_REQUESTS = 64
STREAM_ITERS = 50
STREAM_2D_SIZES = (255, 383, 511, 767, 1023, 1535, 2047)
STREAM_2D_ANGLES = (180, 360, 720, 1080, 1800)
STREAM_3D_DIMS = ((15, 255, 255), (21, 383, 383), (31, 511, 511))
STREAM_3D_TILTS = (20, 25, 30, 35, 40, 45)
STREAM_3D_ANGLES = 360


def stream_requests(count=STREAM_REQUESTS, seed=3000):
    """The served request mix: 70 % 2D slices (n from a ladder of odd sizes whose
    steps are about x1.4, so a uniform pick is log-uniform over 255..2047;
    180..1800 angles over [0, pi)), 30 % laminography volumes (three sizes with a
    detector of the volume's width, 360 angles over [0, 2 pi), tilt 20..45
    degrees in 5-degree steps so that geometries repeat), CG or Split-Bregman
    with equal odds.  Returns (arrival time at rate 1, key, method); at rate r
    the arrival times are these divided by r, so every rate sees the same
    requests in the same order (open-loop Poisson arrivals)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for _ in range(count):
        t += rng.exponential(1.0)
        if rng.random() < 0.7:
            key = ("2d", STREAM_2D_SIZES[rng.integers(len(STREAM_2D_SIZES))],
                   STREAM_2D_ANGLES[rng.integers(len(STREAM_2D_ANGLES))])
        else:
            key = ("3d", STREAM_3D_DIMS[rng.integers(len(STREAM_3D_DIMS))],
                   STREAM_3D_TILTS[rng.integers(len(STREAM_3D_TILTS))])
        out.append((t, key, "cg" if rng.random() < 0.5 else "sb"))
    return out


class StreamInputs:
    """Host inputs per geometry of the stream, built once: one seeded phantom per
    size, forward-projected on the GPU for each angle set or tilt, plus 1 %
    noise (2D sinograms normalised by their maximum, as the reference's
    prepare_sinogram does; 3D projections raw, MBIR normalises them)."""

    def __init__(self, lc):
        self.lc = lc
        self.phantoms = {}
        self.inputs = {}

    def get(self, key):
        if key in self.inputs:
            return self.inputs[key]
        import torch
        from laminocam_b200 import synthetic as S
        lc = self.lc
        if key[0] == "2d":
            _, n, nth = key
            if n not in self.phantoms:
                self.phantoms[n] = S.ellipse_phantom(n, 10, 1000 + n)
            th = np.arange(nth) * np.pi / nth
            s = lc.forward2d(torch.as_tensor(self.phantoms[n][None], device="cuda"),
                             lc.PolarGrid2D(th, n)).cpu().numpy()
            s = S.add_noise(s, NOISE, 2000 + n + nth)
            val = (np.ascontiguousarray(s / s.max(), dtype=np.float32), th)
        else:
            _, dims, tilt = key
            if dims not in self.phantoms:
                self.phantoms[dims] = S.ellipsoid_phantom(dims, N_ELLIPSOIDS, 1000 + dims[0])
            th = np.arange(STREAM_3D_ANGLES) * 2 * np.pi / STREAM_3D_ANGLES
            gam = -tilt * np.pi / 180.0
            pg = lc.PolarGrid(th, np.full(len(th), gam), np.zeros(len(th)), dims[1], dims[2])
            p = lc.forward(torch.as_tensor(self.phantoms[dims], device="cuda"), pg)
            p = p + NOISE * p.max() * torch.randn(
                p.shape, device="cuda", generator=torch.Generator("cuda").manual_seed(2000 + tilt))
            val = (np.ascontiguousarray(p.cpu().numpy(), dtype=np.float32), th, gam)
            del pg
        self.inputs[key] = val
        return val


def stream_params(lc, key, method, plain, iters=STREAM_ITERS):
    """Plain: FP32 scalars, a host check of the solver state after every
    iteration (a tolerance of 1e-30 keeps the check without ever stopping), no
    graphs, the reference's residual schedule.  Served: FP64 scalars, a fixed
    count, CUDA-graph iterations, the operator product carried for 16 outer
    iterations."""
    dims = (1, key[1], key[1]) if key[0] == "2d" else key[1]
    stop = 1e-30 if plain else 0.0
    common = dict(recon_dims=dims, max_iters=iters, inner_iters=1, lam=LAM, mu=MU,
                  fp32_scalars=plain, use_graph=not plain, poll_every=1 if plain else 8)
    if method == "cg":
        return lc.ReconParams(regularizer="unconstrained", tol=stop, xtol=0.0, **common)
    return lc.ReconParams(regularizer="split_bregman", tol=0.0, xtol=stop,
                          residual_refresh=1 if plain else 16, **common)


def serving_stream(lc, workers=32, count=STREAM_REQUESTS, rates=STREAM_RATES):
    """The served request stream against plain sequential GPU solves, both
    open-loop at the same Poisson arrival times.  Plain: one request at a time
    through MBIR2D / MBIR in arrival order (a request waits for the previous
    one), each building its own PSF.  Served: each request submitted to one
    long-lived server at its arrival time; the server's PSF cache is cleared
    before each rate, so hits come only from geometries repeated within the
    stream.  Wall clock, host buffers in and out; recons/s = requests / (end of
    the last request - start), latency = end - arrival."""
    import torch
    from oracle import oracle as O
    reqs = stream_requests(count)
    data = StreamInputs(lc)
    for _, key, _ in reqs:
        data.get(key)
    torch.cuda.synchronize()

    def plain_solve(key, method, iters=STREAM_ITERS):
        d = data.get(key)
        prm = stream_params(lc, key, method, True, iters)
        if key[0] == "2d":
            return lc.MBIR2D(d[0], d[1], prm)
        return lc.MBIR([lc.Dataset(d[0], d[1], d[2], 0.0)], prm)

    def submit(sv, key, method, iters=STREAM_ITERS):
        d = data.get(key)
        prm = stream_params(lc, key, method, False, iters)
        if key[0] == "2d":
            return sv.submit2d(d[0], d[1], prm)
        return sv.submit3d([lc.Dataset(d[0], d[1], d[2], 0.0)], prm)

    # untimed: one iteration of every geometry and method in both forms fills
    # the FFT launch-tuner cache (shared by the process) and grows every
    # worker's buffers, so neither form pays first-use costs in the timed runs
    shapes = sorted({(k, m) for _, k, m in reqs}, key=str)
    for k, m in shapes:
        plain_solve(k, m, 1)
    out = {"workload": f"{count} requests, Poisson arrivals (seed 3000): 70 % 2D slices n in "
                       f"{list(STREAM_2D_SIZES)}, angles in {list(STREAM_2D_ANGLES)}; 30 % laminography "
                       f"volumes {[list(d) for d in STREAM_3D_DIMS]}, tilt {list(STREAM_3D_TILTS)} deg, "
                       f"{STREAM_3D_ANGLES} angles; CG {STREAM_ITERS} iterations or Split-Bregman "
                       f"{STREAM_ITERS} outer x 1 inner (lambda {LAM}, mu {MU}), 50/50; 1 % noise",
           "distinct_geometries": len({k for _, k, _ in reqs}),
           "timing": "wall clock, host buffers in and out, open loop", "rates": []}
    with lc.Server(workers=workers) as sv:
        for _ in range(2):
            ids = [submit(sv, k, m, 1) for k, m in shapes]
            for j in ids:
                sv.wait(j, 600)
        for rate in rates:
            # plain, in arrival order
            t0 = time.perf_counter()
            lat, plain_out, service = [], [], {}
            for u, key, method in reqs:
                arr = t0 + u / rate
                now = time.perf_counter()
                if now < arr:
                    time.sleep(arr - now)
                a = time.perf_counter()
                plain_out.append(plain_solve(key, method))
                b = time.perf_counter()
                lat.append((b - arr) * 1e3)
                cat = f"{key[0]}_{key[1] if key[0] == '2d' else key[1][0]}_{method}"
                c = service.setdefault(cat, [0, 0.0])
                c[0] += 1
                c[1] += (b - a) * 1e3
            t_plain = time.perf_counter() - t0
            # served
            sv.clear_psf_cache()
            sv.reset_stats()
            t0 = time.perf_counter()
            subs = []
            for u, key, method in reqs:
                arr = t0 + u / rate
                now = time.perf_counter()
                if now < arr:
                    time.sleep(arr - now)
                subs.append((submit(sv, key, method), time.perf_counter() - arr))
            res = [sv.wait(j, 600) for j, _ in subs]
            t_served = time.perf_counter() - t0
            st = sv.stats()
            slat = [lag * 1e3 + r.latency_ms for (_, lag), r in zip(subs, res)]
            diffs = [O.rel_l2(r.recon, p) for r, p in zip(res, plain_out)]

            def by_class(lats, kind):
                v = [x for x, (_, key, _) in zip(lats, reqs) if key[0] == kind]
                return {"p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99))} if v else None
            out["rates"].append({
                "rate_req_s": rate,
                "plain": {"recons_per_s": count / t_plain, "seconds": t_plain,
                          "latency_ms_p50": float(np.percentile(lat, 50)),
                          "latency_ms_p99": float(np.percentile(lat, 99)),
                          "latency_ms_2d": by_class(lat, "2d"), "latency_ms_3d": by_class(lat, "3d"),
                          "service_ms_by_kind": {k: {"requests": v[0], "total_ms": round(v[1], 1)}
                                                 for k, v in sorted(service.items())}},
                "served": {"recons_per_s": count / t_served, "seconds": t_served,
                           "latency_ms_p50": float(np.percentile(slat, 50)),
                           "latency_ms_p99": float(np.percentile(slat, 99)),
                           "latency_ms_2d": by_class(slat, "2d"), "latency_ms_3d": by_class(slat, "3d"),
                           "backfilled": st["backfilled"],
                           "peak_running": st["peak_running"],
                           "peak_admitted_gb": st["peak_admitted_bytes"] / 1e9,
                           "psf_hits": st["psf_hits"], "psf_misses": st["psf_misses"],
                           "psf_hit_rate": st["psf_hits"] / max(1, st["psf_hits"] + st["psf_misses"])},
                "speedup": t_plain / t_served,
                "max_rel_l2_served_vs_plain": {
                    m: max([d for d, (_, _, mm) in zip(diffs, reqs) if mm == m] or [0.0])
                    for m in ("cg", "sb")},
            })
        # the error of both forms against the FP64 oracle on small jobs of the
        # stream's two solver kinds
        from laminocam_b200 import synthetic as S
        th1 = np.arange(60) * np.pi / 60
        s1 = lc.forward2d(S.ellipse_phantom(63, 10, 4000)[None], lc.PolarGrid2D(th1, 63)).cpu().numpy()
        s1 = np.ascontiguousarray(S.add_noise(s1, NOISE, 4001), dtype=np.float32)
        s1 /= s1.max()
        key1 = ("2d", 63, 60)
        data.inputs[key1] = (s1, th1)
        err = {}
        for m in ("cg", "sb"):
            xs = sv.wait(submit(sv, key1, m), 600).recon
            xp = plain_solve(key1, m)
            xo = O.mbir2d(s1.astype(np.float64), th1, (1, 63, 63), method=m, max_iters=STREAM_ITERS,
                          tol=0, xtol=0, lam=LAM, mu=MU)
            err[m] = {"served": O.rel_l2(xs, xo), "plain": O.rel_l2(xp, xo)}
        out["rel_l2_vs_fp64_oracle_n63"] = err
    return out


def run_reference(args, rank, world):
    """The reference arm: the reference's own CPU path (reference_cpu_run) on
    this workload.  A step is one Split-Bregman outer iteration of the
    reference's code at the workload size; the setup (backprojection and PSF)
    runs once before the warm-up and is timed too.  value = 1 / (setup + the
    workload's 100 outer iterations x the mean timed outer iteration): one
    reconstruction's worth of the reference's measured work, in recons/s.
    Under torchrun only rank 0 runs."""
    if rank != 0:
        return
    try:
        r = reference_cpu_run(args.warmup, args.steps, full=args.reference_full)
    except Exception as ex:
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU build failed to run: {ex}"}),
              flush=True)
        return
    v = 1.0 / r["recon_s"]
    sec = float(np.mean(r["outer_s"]))
    line = {"metric": METRIC, "value": v, "unit": "recons/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": CONFIG, "impl": "reference",
            "value_basis": f"1 / (setup + {OUTER} x mean outer iteration); a step is one outer iteration",
            "reference_times_s": {"setup": r["setup_s"], "backproj": r["backproj_s"], "psf": r["psf_s"],
                                  "outer_mean": sec, "outer_steps": [round(t, 3) for t in r["outer_s"]],
                                  "full_reconstruction": r["full_s"]},
            "cpu_baseline": {"value": v, "unit": "recons/s", "cores": r["cores"], "kind": "reference",
                             "sample": f"the reference's own sources in float on self-written multithreaded "
                                       f"FFTW/FINUFFT stand-ins (FINUFFT tol 5e-4), {r['cores']} threads: "
                                       f"setup once, {args.warmup} untimed and {args.steps} timed outer "
                                       f"iterations"},
            "e2e": {"value": v, "unit": "recons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def kernel_case(case: str, reps: int):
    """Reduced cases for profiler captures of one kernel family; prints
    timings, not a benchmark line.  At the workload's padded volume
    [29, 721, 721] (P = [64, 1458, 1458]):
      toeplitz       PSF from the workload's 360 angles, then `reps` A^T A applies
      split_bregman  PSF from 12 of the angles (cheap to build), then
                     Split-Bregman with `reps` outer iterations, one CG each
    and for the 2D paths:
      batch          the 64-job uneven mix through lc_mbir2d_batch with `reps`
                     CG iterations (no graph, so each launch is visible)
      noalloc        `reps` allocation-free Toeplitz applies of 2 slices of
                     1023 x 1023 (P = 2048)"""
    import torch
    import laminocam_b200 as lc
    if case == "batch":
        jobs = mix_jobs(lc)
        p = lc.ReconParams(regularizer="unconstrained", recon_dims=(1, 1, 1), max_iters=reps, tol=0.0, xtol=0.0)
        lc.MBIR2D_batch(jobs, p)
        torch.cuda.synchronize()
        t0 = time.time()
        lc.MBIR2D_batch(jobs, p)
        print(json.dumps({"kernel_case": case, "jobs": len(jobs), "iters": reps,
                          "ms": (time.time() - t0) * 1e3}), flush=True)
        return
    if case == "noalloc":
        import ctypes as C
        n, nth, ns = 1023, 720, 2
        th = np.arange(nth) * np.pi / nth
        psf = lc.PointSpreadFunction2D(lc.PolarGrid2D(th, n), n, ns)
        spec = torch.as_tensor(psf.spectrum(), device="cuda").contiguous()
        x = torch.rand((ns, n, n), device="cuda", generator=torch.Generator("cuda").manual_seed(5))
        y = torch.empty_like(x)
        lib = lc._lib.load()
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream or 1)
        assert lib.lc_sysmat2d_toeplitz_noalloc(None, None, 0, None, None, 0, 0) == 0
        torch.cuda.synchronize()
        t0 = time.time()
        for _ in range(reps):
            rc = lib.lc_sysmat2d_toeplitz_noalloc(stream, C.c_void_p(spec.data_ptr()), psf.P[2],
                                                  C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), ns, n)
            assert rc == 0, rc
        torch.cuda.synchronize()
        print(json.dumps({"kernel_case": case, "P": psf.P[2], "reps": reps,
                          "ms_per_rep": (time.time() - t0) * 1e3 / reps}), flush=True)
        return
    n1, n = 29, 721
    nth = NANGLES if case == "toeplitz" else 12
    th = np.arange(nth) * 2 * np.pi / nth
    pg = lc.PolarGrid(th, np.full(nth, -GAMMA_DEG * np.pi / 180.0), np.zeros(nth), DET[0], DET[1])
    psf = lc.PointSpreadFunction(pg, (n1, n, n))
    x = torch.rand((n1, n, n), device="cuda", generator=torch.Generator("cuda").manual_seed(5))
    torch.cuda.synchronize()
    t0 = time.time()
    if case == "toeplitz":
        for _ in range(reps):
            psf.convolve(x)
    else:
        lc.split_bregman(psf, x, torch.zeros_like(x), LAM, MU, reps, 1, 0.0, 0.0)
    torch.cuda.synchronize()
    print(json.dumps({"kernel_case": case, "P": list(psf.P), "reps": reps,
                      "ms_per_rep": (time.time() - t0) * 1e3 / reps}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--clock-interval", type=float, default=0.25,
                    help="seconds between clock samples during the timed region")
    ap.add_argument("--residual-refresh", type=int, default=16,
                    help="Split-Bregman: recompute A x of the warm-started residual every this many "
                         "outer iterations (1: every one, the reference's schedule); carried by the "
                         "CG updates in between")
    ap.add_argument("--no-mix", action="store_true",
                    help="skip the served-vs-plain 64-job 2D mix")
    ap.add_argument("--no-stream", action="store_true",
                    help="skip the served-vs-plain Poisson request stream")
    ap.add_argument("--stream-only", action="store_true",
                    help="run only the served-vs-plain Poisson request stream and print its figures")
    ap.add_argument("--stream-requests", type=int, default=STREAM_REQUESTS,
                    help="requests per arrival rate of the request stream")
    ap.add_argument("--small", action="store_true",
                    help="reduced case for profiler captures: recon_dims [15,255,255], 180 angles, "
                         "255x255 detector, 5 outer iterations (not a benchmark line)")
    ap.add_argument("--kernel-case", choices=["toeplitz", "split_bregman", "batch", "noalloc"],
                    help="reduced case for a profiler capture of one kernel family (not a benchmark line)")
    ap.add_argument("--reps", type=int, default=3, help="applies or outer iterations of --kernel-case")
    ap.add_argument("--precision-study", action="store_true",
                    help="run the precision study (2047x2047 slice, 1800 angles; default FP32 path with FP64 "
                         "PSF and scalars, all-FP32, the reference's float path) against the FP64 oracle and "
                         "print its JSON line (a few minutes of host time for the oracle)")
    ap.add_argument("--reference-full", action="store_true",
                    help="with --impl reference: also run one complete reconstruction of the reference's "
                         "code (tomocam::MBIR, 100 outer iterations) and report its time beside the "
                         "sampled value")
    args = ap.parse_args()
    if args.kernel_case:
        return kernel_case(args.kernel_case, args.reps)
    if args.small:
        global RECON_DIMS, NANGLES, DET, OUTER, N_ELLIPSOIDS
        RECON_DIMS, NANGLES, DET, OUTER, N_ELLIPSOIDS = (15, 255, 255), 180, (255, 255), 5, 10
        CONFIG.update({"workload": "small profiling case (not the benchmark workload)",
                       "recon_dims": list(RECON_DIMS), "padded_dims": [21, 359, 359],
                       "angles": NANGLES, "detector": list(DET), "outer_iters": OUTER})
        args.no_cpu_baseline = True
        args.no_mix = True
        args.no_stream = True

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.precision_study:
        import laminocam_b200 as lc
        if rank == 0:
            print(json.dumps({"precision_study": precision_study(lc)}), flush=True)
        return
    if args.stream_only:
        import laminocam_b200 as lc
        if rank == 0:
            print(json.dumps({"serving_stream": serving_stream(lc, count=args.stream_requests)}),
                  flush=True)
        return

    import ctypes as C

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    import laminocam_b200 as lc
    from laminocam_b200 import _lib

    ctx = lc.Context.default(local)
    lib = ctx.lib
    theta, gamma = geometry()
    vol, dproj = make_projections(lc)
    nth, nr, nc = dproj.shape
    gam = np.full(nth, gamma)
    bet = np.zeros(nth)
    # the outer iterations replay as a CUDA graph (the first one runs eagerly)
    params = lc.ReconParams(regularizer="split_bregman", recon_dims=RECON_DIMS, max_iters=OUTER,
                            inner_iters=1, lam=LAM, mu=MU, tol=1e-5, xtol=0.0, use_graph=True,
                            residual_refresh=args.residual_refresh).to_c()
    CONFIG["residual_refresh"] = args.residual_refresh
    rd = (C.c_int * 3)(*RECON_DIMS)
    _, tp = lc._dptr(theta)
    _, gp = lc._dptr(gam)
    _, bp = lc._dptr(bet)
    th_keep = (np.ascontiguousarray(theta), np.ascontiguousarray(gam), np.ascontiguousarray(bet))
    tp = th_keep[0].ctypes.data_as(C.POINTER(C.c_double))
    gp = th_keep[1].ctypes.data_as(C.POINTER(C.c_double))
    bp = th_keep[2].ctypes.data_as(C.POINTER(C.c_double))
    drecon = torch.empty(RECON_DIMS, dtype=torch.float32, device="cuda")
    host_proj = torch.empty(dproj.shape, dtype=torch.float32, pin_memory=True)
    host_proj.copy_(dproj.cpu())
    host_recon = torch.empty(RECON_DIMS, dtype=torch.float32, pin_memory=True)
    stats = _lib.SolverStats()

    def step_device():
        ctx.sync_stream()
        rc = lib.lc_mbir3d_device(ctx.handle, C.c_void_p(dproj.data_ptr()), nth, nr, nc, tp, gp, bp,
                                  None, rd, C.byref(params), C.c_void_p(drecon.data_ptr()), C.byref(stats))
        if rc:
            raise RuntimeError(lib.lc_last_error(ctx.handle).decode())

    def step_e2e():
        ctx.sync_stream()
        rc = lib.lc_mbir3d(ctx.handle, C.cast(host_proj.data_ptr(), C.POINTER(C.c_float)), nth, nr, nc,
                           tp, gp, bp, None, rd, C.byref(params),
                           C.cast(host_recon.data_ptr(), C.POINTER(C.c_float)), C.byref(stats))
        if rc:
            raise RuntimeError(lib.lc_last_error(ctx.handle).decode())

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, k):
        lat = []
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            lat.append((a, b))
        e1.record()
        barrier()
        total = e0.elapsed_time(e1)
        lats = [a.elapsed_time(b) for a, b in lat]
        if dist is not None:
            t = torch.tensor([total], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            total = float(t.item())
        return total, lats

    # the clock sampler's NVML set-up runs before the warm-up steps
    clk = ClockSampler(local, args.clock_interval)
    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()

    with clk:
        launches0 = lib.lc_kernel_launches()
        total_ms, lats = timed(step_device, args.steps)
        launches = lib.lc_kernel_launches() - launches0
    value = args.steps * world / (total_ms / 1e3)

    # one more step with per-section CUDA events (not part of the timed region)
    lib.lc_profile_enable(ctx.handle, 1)
    step_device()
    torch.cuda.synchronize()
    entries = (_lib.ProfileEntry * 32)()
    nent = C.c_int()
    lib.lc_profile_read(ctx.handle, entries, 32, C.byref(nent))
    lib.lc_profile_enable(ctx.handle, 0)

    # end to end through the host-buffer API
    step_e2e()
    e2e_ms, _ = timed(step_e2e, args.steps)
    e2e_value = args.steps * world / (e2e_ms / 1e3)

    # roofline of the dominant kernel section
    prof = []
    for i in range(nent.value):
        e = entries[i]
        prof.append({"name": e.name.decode(), "launches": e.count, "total_ms": e.total_ms,
                     "avg_ms": e.total_ms / max(e.count, 1), "gbs": e.bytes / max(e.total_ms, 1e-9) / 1e6,
                     "bytes_per_launch": e.bytes / max(e.count, 1)})
    prof.sort(key=lambda d: -d["total_ms"])
    peak, peak_kind = measured_peak()
    # The Toeplitz apply (A^T A, the per-iteration hot spot) is one unit of five
    # line-FFT launches; it competes with the single sections for "dominant".
    toep = [p for p in prof if p["name"].startswith("toeplitz_")]
    units = [p for p in prof if not p["name"].startswith("toeplitz_") and p["bytes_per_launch"] > 0]
    if toep:
        applies = max(p["launches"] for p in toep)
        tot_ms = sum(p["total_ms"] for p in toep)
        tot_b = sum(p["bytes_per_launch"] * p["launches"] for p in toep)
        units.append({"name": "toeplitz_apply (" + "+".join(p["name"][9:] for p in toep) + ")",
                      "launches": applies, "total_ms": tot_ms, "avg_ms": tot_ms / applies,
                      "gbs": tot_b / tot_ms / 1e6, "bytes_per_launch": tot_b / applies})
    # The roofline object is the section with the most time in the step,
    # one-off sections (the spreading) included; every section is listed in
    # "rooflines".
    dom = max(units, key=lambda d: d["total_ms"]) if units else None
    rooflines = [{"section": u["name"], "launches": u["launches"], "avg_ms": u["avg_ms"],
                  "achieved_gbs": u["gbs"], "frac": u["gbs"] / peak} for u in
                 sorted(units, key=lambda d: -d["total_ms"])]
    roof = None
    if dom:
        traffic = None
        if dom["name"].startswith("toeplitz_apply") and not args.small:
            # DRAM bytes read + written by the five passes of one apply at this
            # workload, from one ncu capture (--kernel-case toeplitz); writes
            # still in L2 when a pass ends are not counted
            traffic = TOEPLITZ_APPLY_DRAM_BYTES
        roof = {"bound": "hbm", "kernel": dom["name"], "achieved": dom["gbs"], "peak": peak,
                "unit": "GB/s", "frac": dom["gbs"] / peak, "peak_source": peak_kind,
                "bytes_per_launch": dom["bytes_per_launch"], "avg_launch_ms": dom["avg_ms"],
                "traffic": traffic}

    # The spreading against its own bound: every cell update of a footprint
    # is two 32-bit shared-memory reductions (the fixed-point words of the
    # real and imaginary parts), and an SM retires about 31 of them per clock
    # (a conflict-free probe measured 30.9).
    spread_roof = None
    sp = next((u for u in units if u["name"] == "nufft_spread"), None)
    if sp and not args.small:
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        mhz = clk.summary().get("sm_mhz") or 1965.0
        w = 7  # ES kernel width at NUFFT tolerance 1e-6
        cells = float(NANGLES) * PADDED_DET[0] * PADDED_DET[1] * w ** 3
        bound_ms = cells * 2.0 / (SHARED_RED_PER_CLK_SM * sms * mhz * 1e6) * 1e3
        spread_roof = {"bound": "shared-memory reductions", "cell_updates": cells,
                       "reductions_per_cell": 2, "peak_reductions_per_clk_per_sm": SHARED_RED_PER_CLK_SM,
                       "bound_ms": bound_ms, "avg_launch_ms": sp["avg_ms"], "frac": bound_ms / sp["avg_ms"],
                       "hbm_gbs": sp["gbs"], "hbm_frac": sp["gbs"] / peak}

    # the same reconstruction with the operator product recomputed in every
    # outer iteration (the reference's schedule): its rate and its relative L2
    # difference from the carried schedule's result
    schedule_check = None
    exact_value = None
    if args.residual_refresh != 1:
        carried = drecon.clone()
        exact_params = lc.ReconParams(regularizer="split_bregman", recon_dims=RECON_DIMS, max_iters=OUTER,
                                      inner_iters=1, lam=LAM, mu=MU, tol=1e-5, xtol=0.0, use_graph=True,
                                      residual_refresh=1).to_c()

        def step_exact():
            ctx.sync_stream()
            rc = lib.lc_mbir3d_device(ctx.handle, C.c_void_p(dproj.data_ptr()), nth, nr, nc, tp, gp, bp,
                                      None, rd, C.byref(exact_params), C.c_void_p(drecon.data_ptr()), None)
            if rc:
                raise RuntimeError(lib.lc_last_error(ctx.handle).decode())

        step_exact()
        torch.cuda.synchronize()
        schedule_check = float(torch.linalg.vector_norm((carried - drecon).double())
                               / torch.linalg.vector_norm(drecon.double()))
        k_exact = max(1, min(args.steps, 5))
        exact_ms, _ = timed(step_exact, k_exact)
        exact_value = k_exact * world / (exact_ms / 1e3)

    serving = None
    if rank == 0 and world == 1 and not args.no_mix:
        try:
            serving = serving_mix(lc)
        except Exception as ex:  # reported, not fatal
            serving = {"error": repr(ex)}

    stream = None
    if rank == 0 and world == 1 and not args.no_stream:
        try:
            stream = serving_stream(lc, count=args.stream_requests)
        except Exception as ex:  # reported, not fatal
            stream = {"error": repr(ex)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline()
        except Exception as ex:  # reported, not fatal
            cpu = {"value": None, "unit": "recons/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {ex}"}

    lats_sorted = sorted(lats)
    line = {
        "metric": METRIC, "value": value, "unit": "recons/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 PSF and solver scalars)",
        "data": "synthetic", "config": CONFIG,
        "latency_ms": {"p50": float(np.percentile(lats_sorted, 50)),
                       "p99": float(np.percentile(lats_sorted, 99)),
                       "steps": [round(v, 2) for v in lats]},
        "e2e": {"value": e2e_value, "unit": "recons/s",
                "h2d_bytes_per_step": int(host_proj.numel() * 4),
                "d2h_bytes_per_step": int(host_recon.numel() * 4)},
        "roofline": roof, "rooflines": rooflines, "kernels": prof[:12], "clocks": clk.summary(),
        "serving": serving, "serving_stream": stream, "gpu_launches": int(launches),
        "cpu_baseline": cpu,
        "spread_roofline": spread_roof,
        "value_reference_schedule": exact_value,
        "solver": {"outer_iters": stats.iters, "cg_iters": stats.cg_iters_total, "dx": stats.dx,
                   "residual_refresh": args.residual_refresh,
                   "rel_l2_vs_exact_residual_schedule": schedule_check},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

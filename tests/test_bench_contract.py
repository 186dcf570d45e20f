"""CPU checks of bench.py: the served request stream's workload (seeded,
70 % slices / 30 % volumes, CG or Split-Bregman with equal odds, the size and
angle ladders) and the reference arm's JSON line, which runs the reference's
own CPU path (oracle/_ref/ref_bench) on the host and needs no GPU."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_stream_requests_are_seeded_and_follow_the_mix():
    a = bench.stream_requests(400)
    b = bench.stream_requests(400)
    assert a == b
    t = np.array([r[0] for r in a])
    assert np.all(np.diff(t) > 0)
    # unit-rate Poisson arrivals: mean gap 1
    assert abs(np.mean(np.diff(np.concatenate([[0.0], t]))) - 1.0) < 0.15
    kinds = [r[1][0] for r in a]
    methods = [r[2] for r in a]
    assert abs(kinds.count("2d") / len(a) - 0.7) < 0.08
    assert abs(methods.count("cg") / len(a) - 0.5) < 0.08
    for _, key, method in a:
        assert method in ("cg", "sb")
        if key[0] == "2d":
            assert key[1] in bench.STREAM_2D_SIZES and key[2] in bench.STREAM_2D_ANGLES
        else:
            assert key[1] in bench.STREAM_3D_DIMS and key[2] in bench.STREAM_3D_TILTS
    # the default stream repeats geometries, so the PSF cache can hit
    keys = [r[1] for r in bench.stream_requests()]
    assert len(set(keys)) < len(keys)


def test_stream_params_forms():
    class FakeLc:
        class ReconParams:
            def __init__(self, **kw):
                self.__dict__.update(kw)

    plain = bench.stream_params(FakeLc, ("3d", (15, 255, 255), 30), "sb", True)
    served = bench.stream_params(FakeLc, ("3d", (15, 255, 255), 30), "sb", False)
    assert plain.recon_dims == (15, 255, 255) and plain.max_iters == bench.STREAM_ITERS
    assert plain.fp32_scalars and not plain.use_graph and plain.poll_every == 1 and plain.xtol > 0
    assert plain.residual_refresh == 1
    assert not served.fp32_scalars and served.use_graph and served.xtol == 0
    cg = bench.stream_params(FakeLc, ("2d", 511, 360), "cg", True)
    assert cg.regularizer == "unconstrained" and cg.recon_dims == (1, 511, 511) and cg.tol > 0


def test_reference_arm_prints_its_line():
    """The reduced profiling case (--small) keeps the reference's CPU run short."""
    from oracle import refrun
    if not refrun.bench_available():
        import pytest
        pytest.skip("oracle/_ref/ref_bench is not built")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "1", "--small"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["value"] > 0 and line["unit"] == "recons/s"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
    t = line["reference_times_s"]
    assert len(t["outer_steps"]) == 2 and t["setup"] > 0
    # value is one reconstruction's worth of the measured work: setup + the
    # workload's outer iterations (100; 5 in the reduced case)
    outer = line["config"]["outer_iters"]
    assert abs(1.0 / line["value"] - (t["setup"] + outer * t["outer_mean"])) < 1e-6 * (1.0 / line["value"])
    assert abs(line["ms_per_step"] - 1e3 * t["outer_mean"]) < 1e-6 * line["ms_per_step"]

"""FP64 PSF generators against the oracle and against each other.

3D, laminography (beta = 0, one tilt gamma for every angle): the kernel
factors as K(k) = D_nx(cg kx - sg ky) * S(sg kx + cg ky, kz) with
S(u, kz) = sum_theta D_ny(cos(theta) u - sin(theta) kz) (include/toeplitz.h
sums the same Dirichlet products angle by angle).  S is band-limited in u,
so the device sums it exactly on a grid of u of spacing 1/32 and interpolates
it with ten points (about 1e-13 of the kernel's peak).  Scans that are not
closed under theta -> -theta, or that mix tilts, keep the direct sum;
LC_PSF_TABLE=0 forces the direct sum everywhere.

2D: the angle sum of each 16-point row segment is split over 1 to 32 lanes
of a warp, by the grid size and angle count, so that small slices fill the
GPU; the cases below reach every split."""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lc(cuda):
    import laminocam_b200 as lc
    return lc


def zero_unpaired(K):
    K = K.copy()
    for ax in range(K.ndim):
        if K.shape[ax] % 2 == 0:
            idx = [slice(None)] * K.ndim
            idx[ax] = 0
            K[tuple(idx)] = 0.0
    return K


@pytest.mark.parametrize("turn,gamma,nth,dims", [
    (np.pi, -20.0, 30, (7, 21, 21)),      # the reference's [-90, 90) scan
    (2 * np.pi, 35.0, 24, (5, 16, 16)),   # a full turn, even sizes
    (np.pi, 0.0, 18, (6, 15, 17)),        # no tilt: u = ky
    (np.pi, -90.0, 18, (4, 13, 13)),      # u = -kx
])
def test_table_against_oracle(lc, turn, gamma, nth, dims):
    th = -turn / 2 + np.arange(nth) * turn / nth
    g = np.full(nth, np.deg2rad(gamma))
    nr, nc = dims[1] + 2, dims[2] + 1
    pg = lc.PolarGrid(th, g, np.zeros(nth), nr, nc)
    K = lc.PointSpreadFunction(pg, dims).kernel()
    want = zero_unpaired(O.psf3d(O.Grid3D(th, g, np.zeros(nth), nr, nc), dims).kernel)
    err = O.rel_l2(K, want)
    peak = np.abs(want).max()
    print("table vs oracle", turn, gamma, err, np.abs(K - want).max() / peak)
    assert err < 1e-11, err
    assert np.abs(K - want).max() < 1e-11 * peak


SCRIPT = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import laminocam_b200 as lc
nth, n, n1 = (int(v) for v in sys.argv[3:6])
th = -np.pi / 2 + np.arange(nth) * np.pi / nth
pg = lc.PolarGrid(th, np.full(nth, -np.deg2rad(30.0)), np.zeros(nth), n, n)
np.save(sys.argv[2], lc.PointSpreadFunction(pg, (n1, n, n)).kernel())
"""


def run_kernel(tmp_path, name, table, nth, n, n1):
    out = str(tmp_path / name)
    env = dict(os.environ, LC_PSF_TABLE="1" if table else "0")
    subprocess.run([sys.executable, "-c", SCRIPT, ROOT, out, str(nth), str(n), str(n1)], check=True, env=env,
                   timeout=600)
    return np.load(out + ".npy")


def test_table_and_direct_sum_against_oracle(tmp_path):
    """90 angles, 48 x 48 detector: both generators against the oracle.  The
    direct sum advances sin(pi u / n) along kx with steps up to 1/2, and near
    a pole of a Dirichlet term the recurrence's ~5e-16 absolute error is
    amplified (about 1e-11 of the peak); the table's recurrences take steps of
    1/32 or less."""
    nth, n, n1 = 90, 48, 7
    th = -np.pi / 2 + np.arange(nth) * np.pi / nth
    want = zero_unpaired(O.psf3d(O.Grid3D(th, np.full(nth, -np.deg2rad(30.0)), np.zeros(nth), n, n),
                                 (n1, n, n)).kernel)
    Kt = run_kernel(tmp_path, "table", True, nth, n, n1)
    Kd = run_kernel(tmp_path, "direct", False, nth, n, n1)
    et, ed = O.rel_l2(Kt, want), O.rel_l2(Kd, want)
    print("table / direct vs oracle", et, ed)
    assert et < 1e-12, et
    assert ed < 5e-11, ed


def test_table_against_direct_sum(tmp_path):
    """180 angles on a 96 x 96 detector: the tabulated kernel against the
    direct angle sum of the same build, over the whole padded grid, within
    the direct sum's own accuracy."""
    Kt = run_kernel(tmp_path, "table", True, 180, 96, 11)
    Kd = run_kernel(tmp_path, "direct", False, 180, 96, 11)
    peak = np.abs(Kd).max()
    err = np.linalg.norm(Kt - Kd) / np.linalg.norm(Kd)
    print("table vs direct", err, np.abs(Kt - Kd).max() / peak)
    assert err < 5e-11, err
    assert np.abs(Kt - Kd).max() < 5e-11 * peak


@pytest.mark.parametrize("n,nth,kind", [
    (63, 300, "uniform"),    # quarter-turn closed (an eighth summed), 32 lanes per segment
    (64, 130, "random"),     # no mirror, even grid, 16 lanes
    (129, 90, "mirror"),     # closed under theta -> pi - theta only, 8 lanes
    (255, 180, "uniform"),   # 16 lanes
    (511, 64, "uniform"),    # few angles: the quads limit the split (8 lanes)
    (255, 40, "random"),     # 4 lanes
    (31, 6, "random"),       # one lane: fewer than two quads
])
def test_2d_kernel_splits_against_oracle(lc, n, nth, kind):
    rng = np.random.default_rng(n + nth)
    if kind == "uniform":
        th = np.arange(nth) * np.pi / nth
    elif kind == "random":
        th = np.sort(rng.uniform(0, np.pi, nth))
    else:
        half = np.sort(rng.uniform(0.01, np.pi / 2 - 0.01, nth // 2))
        th = np.concatenate([half, np.pi - half[::-1]])
    K = lc.PointSpreadFunction2D(lc.PolarGrid2D(th, n), n, 1).kernel()
    want = zero_unpaired(O.psf2d(th, n, n).kernel)
    err = O.rel_l2(K, want)
    print("2D kernel", n, nth, kind, err)
    assert err < 1e-10, err

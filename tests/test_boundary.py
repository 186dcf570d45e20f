"""CPU tests of the drop-in boundary: the shared library loads, exports every
symbol include/laminocam.h declares, and the Python binding table matches."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "laminocam.h")
LIB = os.path.join(ROOT, "laminocam_b200", "liblaminocam_b200.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lc_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        from laminocam_b200 import build
        build.build()
    return ctypes.CDLL(LIB)


def test_header_declares_the_api():
    names = declared_functions()
    for required in ["lc_forward2d", "lc_backproj2d", "lc_psf_create", "lc_sysmat_toeplitz",
                     "lc_cgsolver", "lc_split_bregman", "lc_mbir2d", "lc_mbir3d", "lc_forward3d",
                     "lc_backproj3d"]:
        assert required in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_table_matches_header():
    from laminocam_b200 import _lib
    assert sorted(_lib.SIGNATURES) == declared_functions()


def test_context_create_without_gpu_fails_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib.lc_context_create.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    h = ctypes.c_void_p()
    rc = lib.lc_context_create(0, None, ctypes.byref(h))
    assert rc != 0 and not h.value


def test_server_rejects_bad_parameters_and_missing_gpu(lib):
    from laminocam_b200 import _lib
    L = _lib.load()
    p = _lib.ServerParams()
    L.lc_server_params_default(ctypes.byref(p))
    assert p.workers == 4 and p.psf_cache == 1 and p.hbm_budget_bytes == 0
    h = ctypes.c_void_p()
    bad = _lib.ServerParams()
    ctypes.memmove(ctypes.byref(bad), ctypes.byref(p), ctypes.sizeof(p))
    bad.workers = 0
    assert L.lc_server_create(ctypes.byref(bad), ctypes.byref(h)) == 1 and not h.value
    import torch
    if not torch.cuda.is_available():
        # no device: creation fails with a CUDA status and leaves no handle
        assert L.lc_server_create(ctypes.byref(p), ctypes.byref(h)) == 3 and not h.value
    assert L.lc_server_destroy(None) == 1
    assert L.lc_server_wait(None, 1, 0.0, None, None) == 1


def test_python_api_refuses_to_run_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import laminocam_b200 as lc
    with pytest.raises(lc.LaminocamError):
        lc.Context(0)


def test_defaults_match_reference(lib):
    from laminocam_b200 import _lib
    L = _lib.load()
    p = _lib.SolverParams()
    L.lc_solver_params_default(ctypes.byref(p))
    assert p.max_iters == 50 and p.inner_iters == 1
    assert abs(p.tol - 1e-5) < 1e-12 and abs(p.lambda_ - 0.1) < 1e-7 and abs(p.mu - 10.0) < 1e-7
    r = _lib.ReconParamsC()
    L.lc_recon_params_default(ctypes.byref(r))
    assert abs(r.pad_factor - 1.4142) < 1e-6 and abs(r.nufft_tol - 1e-6) < 1e-18

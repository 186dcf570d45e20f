"""Builds laminocam_b200/liblaminocam_b200.so from csrc/*.cu for sm_100a.

Run ``python -m laminocam_b200.build`` (or ``__graft_entry__.build()``).  Objects go
to ``laminocam_b200/_build/``; the shared library is placed next to this file so
that it travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblaminocam_b200.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-O3", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp"))]
    deps.append(os.path.join(ROOT, "include", "laminocam.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, extra) -> str:
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    if _stale(obj, src):
        cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if r.stderr.strip() and os.environ.get("LC_BUILD_VERBOSE"):
            print(r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False, extra=()) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, list(extra)), srcs))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    build_drivers()
    if verbose:
        print(LIB)
    return LIB


DRIVERS = os.path.join(HERE, "drivers")
BIN = os.path.join(HERE, "bin")
DRIVER_COMMON = ["lc_toml.cpp", "lc_io.cpp", "lc_config.cpp"]
EXECUTABLES = {"recon_lamino": DRIVER_COMMON + ["recon_lamino.cpp"],
               "recon_tomo": DRIVER_COMMON + ["recon_tomo.cpp"],
               "forward_scalar": ["lc_toml.cpp", "lc_io.cpp", "forward_scalar.cpp"],
               "lc_convert": ["lc_io.cpp", "lc_convert.cpp"]}
# drivers that also call the CUDA runtime (device buffers of their own)
CUDART_DRIVERS = {"forward_scalar"}


def host_cxx() -> str:
    for cand in (os.environ.get("HOSTCXX"), shutil.which("g++"), "/usr/bin/g++"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def build_drivers() -> None:
    """Builds the host-side drivers (plain C++17 over the C ABI) into bin/."""
    os.makedirs(BIN, exist_ok=True)
    deps = [os.path.join(DRIVERS, f) for f in os.listdir(DRIVERS)] + [os.path.join(ROOT, "include", "laminocam.h")]
    newest = max(os.path.getmtime(d) for d in deps)
    for exe, srcs in EXECUTABLES.items():
        out = os.path.join(BIN, exe)
        if os.path.exists(out) and os.path.getmtime(out) >= max(newest, os.path.getmtime(LIB)):
            continue
        cmd = [host_cxx(), "-std=c++17", "-O2", "-Wall", "-o", out,
               *[os.path.join(DRIVERS, s) for s in srcs]]
        if exe != "lc_convert":
            cmd += ["-L", HERE, "-llaminocam_b200", "-Wl,-rpath,$ORIGIN/.."]
        if exe in CUDART_DRIVERS:
            cuda = os.path.dirname(os.path.dirname(os.path.realpath(nvcc())))
            cmd += ["-I", os.path.join(cuda, "include"), "-L", os.path.join(cuda, "lib64"), "-lcudart",
                    "-Wl,-rpath," + os.path.join(cuda, "lib64")]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"building {exe} failed:\n{r.stdout}\n{r.stderr}")


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])

"""Build libwilson_sm100.so in-tree with nvcc for sm_100a.

    python -m jaxqft_b200.build          (or jaxqft_b200.build.build())
    python -m jaxqft_b200.build --check  (libwilson_sm100_check.so, device-side index checks)

The library is written next to this file so that it travels with the source
tree; nothing is installed into site-packages.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libwilson_sm100.so")
SOURCES = ["wl_api.cu"]
HEADERS = ["wl_common.cuh", "wl_hop.cuh", "wl_hop_fast.cuh", "wl_site.cuh", "wl_force.cuh", "wl_gauge.cuh",
           "wl_meas.cuh", "wl_rowhop.cuh", "wl_refsite.cuh", "wl_reftile.cuh", "wl_rng.cuh", "wl_blas.cuh",
           "wl_hop_mma.cuh"]
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
    "-Xptxas", "-O3",
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libwilson_sm100.so")


CHECK_LIB = os.path.join(HERE, "libwilson_sm100_check.so")
CHECK_DEFINES = ["-DWL_BOUNDS_CHECK=1"]  # device-side index checks (see wl_common.cuh)


def _stale(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, "wilson_sm100.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _nvcc_cmd(lib: str, extra=()) -> list:
    return [nvcc(), *NVCC_FLAGS, *extra, "-I", INCLUDE, "-o", lib + ".tmp"] + [os.path.join(CSRC, f) for f in SOURCES]


def _finish(lib: str, res_code: int, out: str, verbose: bool) -> str:
    if res_code != 0:
        sys.stderr.write(out)
        raise RuntimeError(f"nvcc failed building {os.path.basename(lib)}")
    if verbose and out:
        sys.stderr.write(out)
    os.replace(lib + ".tmp", lib)
    return lib


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    """The release library libwilson_sm100.so."""
    if not force and not _stale(LIB):
        return LIB
    cmd = _nvcc_cmd(LIB, extra)
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    return _finish(LIB, res.returncode, res.stdout + res.stderr, verbose)


def build_check(force: bool = False, verbose: bool = False) -> str:
    """The checking library libwilson_sm100_check.so (same sources, WL_BOUNDS_CHECK=1)."""
    if not force and not _stale(CHECK_LIB):
        return CHECK_LIB
    cmd = _nvcc_cmd(CHECK_LIB, CHECK_DEFINES)
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    return _finish(CHECK_LIB, res.returncode, res.stdout + res.stderr, verbose)


def build_all(force: bool = False, verbose: bool = False) -> None:
    """Both libraries, the two nvcc runs in parallel."""
    jobs = []
    for lib, extra in ((LIB, ()), (CHECK_LIB, CHECK_DEFINES)):
        if force or _stale(lib):
            cmd = _nvcc_cmd(lib, extra)
            if verbose:
                print(" ".join(cmd), flush=True)
            jobs.append((lib, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for lib, proc in jobs:
        out, _ = proc.communicate()
        _finish(lib, proc.returncode, out, verbose)


if __name__ == "__main__":
    if "--check" in sys.argv:
        print(build_check(force="--force" in sys.argv, verbose=True))
    else:
        build(force="--force" in sys.argv, verbose=True,
              extra=(["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else []))
        print(LIB)

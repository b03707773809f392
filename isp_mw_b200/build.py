"""Build the B200 BM3D library (``isp_mw_b200/lib/libisp_mw_b200.so``).

nvcc compiles every ``csrc/*.cu`` (in parallel, one process per unit) for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``) and links one shared library exporting the C
ABI declared in ``include/bm3d_b200.h``. The library is built in-tree so it
ships with the repository snapshot; nothing is installed into site-packages.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libisp_mw_b200.so")
CLI = os.path.join(LIBDIR, "isp_mw")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(CLI):
        return True
    t = min(os.path.getmtime(LIB), os.path.getmtime(CLI))
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(
        os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.h")) + glob.glob(
        os.path.join(ROOT, "include", "bm3d_b200", "*.hpp")) + glob.glob(
        os.path.join(PKG, "cli", "*.cpp"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile the library if any source is newer than it; return its path."""
    if not force and not ptxas_info and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    jobs = []
    for src in sources():
        obj = os.path.join(LIBDIR, os.path.basename(src)[:-3] + ".o")
        cmd = [NVCC] + NVCC_FLAGS + ["-I", os.path.join(ROOT, "include"), "-I", CSRC,
                                     "-c", src, "-o", obj]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        jobs.append((cmd, obj))
    # one nvcc per translation unit, in parallel
    workers = max(1, min(len(jobs), os.cpu_count() or 1))
    with ThreadPoolExecutor(workers) as pool:
        results = list(pool.map(
            lambda j: subprocess.run(j[0], stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                     text=True), jobs))
    failed = False
    for (cmd, _), r in zip(jobs, results):
        if r.stdout and (verbose or ptxas_info or r.returncode != 0):
            print(r.stdout, end="", flush=True)
        failed |= r.returncode != 0
    if failed:
        raise subprocess.CalledProcessError(1, "nvcc")
    objs = [obj for _, obj in jobs]
    tmp = LIB + ".tmp"
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "--cudart", "static",
           "-o", tmp] + objs
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    build_cli(verbose)
    return LIB


def build_cli(verbose: bool = False) -> str:
    """The command-line front end (``lib/isp_mw``), linked against the library."""
    src = os.path.join(PKG, "cli", "isp_mw.cpp")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), src,
           "-L", LIBDIR, "-lisp_mw_b200", "-Wl,-rpath,$ORIGIN", "-o", CLI]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return CLI


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)

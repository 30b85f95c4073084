"""Build the sm_100a shared libraries in-tree (pivtools_b200/lib/).

Each reference library name gets its own shared object with the same exported
C symbols: libbulkxcorr2d.so, libfusedwarp.so, libkspacefit.so.  nvcc
cross-compiles on a machine without a GPU; the host-only LaVision codec library
(libpivb_lavision.so) is built with the system C++ compiler.
"""

from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(ROOT, "csrc")
LIBDIR = os.path.join(PKG, "lib")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-shared", "-cudart", "shared",
]

# library -> translation unit
TARGETS = {
    "libbulkxcorr2d.so": "bulkxcorr2d.cu",
    "libfusedwarp.so": "fusedwarp.cu",
    "libkspacefit.so": "kspacefit.cu",
    "libpivb_pass.so": "passglue.cu",
    "libpivb_dft.so": "dftcorr.cu",
    "libpivb_lavision.so": "lavision_codecs.cpp",
}

# host-only translation units: the system C++ compiler, zlib
HOST_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-shared"]
HOST_LIBS = ["-lz", "-pthread"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.isfile(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(out: str, srcs: list[str]) -> bool:
    if not os.path.isfile(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build(force: bool = False, verbose: bool = False, only: list[str] | None = None) -> list[str]:
    """Compile every target whose sources changed (the targets in parallel);
    return the paths built."""
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(LIBDIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    jobs = []
    for lib, tu in TARGETS.items():
        if only and lib not in only:
            continue
        src = os.path.join(CSRC, tu)
        if not os.path.isfile(src):
            continue
        out = os.path.join(LIBDIR, lib)
        if not force and not _stale(out, [src] + headers):
            continue
        jobs.append((src, out))

    def one(job):
        src, out = job
        if src.endswith(".cpp"):
            cmd = [os.environ.get("CXX_HOST", "g++"), *HOST_FLAGS, "-o", out + ".tmp", src, *HOST_LIBS]
        else:
            cmd = [_nvcc(), *NVCC_FLAGS, "-o", out + ".tmp", src]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        os.replace(out + ".tmp", out)
        return out

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        return list(ex.map(one, jobs))


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv, verbose=True):
        print("built", p)

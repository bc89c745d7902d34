"""Build the CUDA library ``eulerianfsi_b200/libefsi.so`` for sm_100a with nvcc.

    python -m eulerianfsi_b200.build [--force]

The library is built in-tree so that it travels with the repository; there is no
JIT path and no CPU fallback.  Freshness is decided by content, not by file times:
a SHA-256 over every source, header and the nvcc command line is stored beside the
library (``libefsi.so.stamp``), and a library whose stamp does not match the current
sources (a copy built from another revision, for example) is rebuilt.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libefsi.so")
STAMP = OUT + ".stamp"
SOURCES = ["efsi_solvers.cu", "efsi_spectral.cu", "efsi_ops.cu", "efsi_adjoint.cu", "efsi_phase.cu", "efsi_diag.cu",
           "efsi_api.cu"]
HEADERS = ["efsi_common.cuh", "efsi_device.cuh", "efsi_kernels.cuh", "efsi_solvers.cuh", "efsi_diag.cuh",
           "efsi_adjoint.cuh"]
PUBLIC_HEADER = os.path.join(os.path.dirname(HERE), "include", "efsi.h")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "-diag-suppress", "177"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _inputs() -> list[str]:
    return [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [PUBLIC_HEADER]


def source_hash() -> str:
    """SHA-256 over the build inputs (names and bytes) and the compiler flags."""
    h = hashlib.sha256()
    h.update(" ".join(GENCODE + FLAGS).encode())
    for path in _inputs():
        h.update(os.path.basename(path).encode())
        with open(path, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def stale() -> bool:
    if not (os.path.exists(OUT) and os.path.exists(STAMP)):
        return True
    with open(STAMP) as f:
        return f.read().strip() != source_hash()


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return OUT
    digest = source_hash()
    build_dir = os.path.join(HERE, "_build")
    os.makedirs(build_dir, exist_ok=True)

    def object_hash(src: str) -> str:  # the source, every header and the flags
        h = hashlib.sha256()
        h.update(" ".join(GENCODE + FLAGS).encode())
        for path in [os.path.join(CSRC, src)] + _inputs()[len(SOURCES):]:
            with open(path, "rb") as f:
                h.update(f.read())
        return h.hexdigest()

    def compile_one(src: str) -> str:
        obj = os.path.join(build_dir, src.replace(".cu", ".o"))
        digest_o = object_hash(src)
        try:  # an object built from the same inputs is reused
            with open(obj + ".stamp") as f:
                if not force and f.read().strip() == digest_o and os.path.exists(obj):
                    return obj
        except OSError:
            pass
        cmd = [nvcc(), *GENCODE, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        with open(obj + ".stamp", "w") as f:
            f.write(digest_o + "\n")
        return obj

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as pool:
        objs = list(pool.map(compile_one, SOURCES))
    tmp = OUT + ".tmp"
    cmd = [nvcc(), *GENCODE, "-shared", "-o", tmp, *objs, "-Xcompiler", "-fPIC"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    with open(STAMP, "w") as f:
        f.write(digest + "\n")
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
